// Grid set-up: twiddle and wavenumber tables, dealiasing cut-offs, buffers.
#include <cmath>
#include <cstring>
#include <mutex>
#include "plan.h"
#include "tma.cuh"

namespace tara {

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }

bool supported_length(int n) {
  switch (n) {
    case 16: case 32: case 64: case 128: case 256: case 384: case 512: case 1024: case 2048:
    case 4096:
      return true;
    default:
      return false;
  }
}

// e^{-2 pi i m/L}: reduce m/L to [0, 1/8] by the symmetries of sin/cos so
// that every table entry is computed from an angle <= pi/4 in long double
// and multiples of pi/4 come out exact.
void twiddle(long m, long L, long double& c, long double& s) {
  m %= L;
  if (m < 0) m += L;
  // angle a = 2 pi m / L; work with 8m/L to find the octant
  long n8 = 8 * m;
  long oct = n8 / L;          // 0..7
  long rem = n8 - oct * L;    // 8m - oct*L, in [0, L)
  const long double pi = 3.141592653589793238462643383279502884L;
  // theta in [0, pi/4): a = oct*pi/4 + rem*pi/(4L)
  long double th, cth, sth;
  // use the reflected angle in odd octants so that the argument stays <= pi/4
  bool odd = oct & 1;
  if (odd) th = (long double)(L - rem) * pi / (4.0L * (long double)L);
  else th = (long double)rem * pi / (4.0L * (long double)L);
  cth = cosl(th);
  sth = sinl(th);
  if (rem == 0 && !odd) { cth = 1; sth = 0; }
  long double ca, sa;  // cos(a), sin(a)
  switch (oct) {
    case 0: ca = cth; sa = sth; break;               // a = th
    case 1: ca = sth; sa = cth; break;               // a = pi/2 - th
    case 2: ca = -sth; sa = cth; break;              // a = pi/2 + th
    case 3: ca = -cth; sa = sth; break;              // a = pi - th
    case 4: ca = -cth; sa = -sth; break;             // a = pi + th
    case 5: ca = -sth; sa = -cth; break;             // a = 3pi/2 - th
    case 6: ca = sth; sa = -cth; break;              // a = 3pi/2 + th
    default: ca = cth; sa = -sth; break;             // a = 2pi - th
  }
  c = ca;
  s = -sa;  // e^{-i a}
}

void wavenumbers(int Nx, int Ny, double Lx, double Ly, double pi, std::vector<double>& kx,
                 std::vector<double>& ky, std::vector<int>& cut) {
  const int Nh = Nx / 2 + 1;
  kx.resize(Nh);
  ky.resize(Ny);
  cut.resize(Ny);
  // kx = 2.0d0*pi*dfloat(i-1)/Lx ; ky = 2.0d0*pi*dfloat(j-1)/Ly (j <= Ny/2),
  // 2.0d0*pi*dfloat((j-1)-Ny)/Ly (j > Ny/2)      (src/derive2coh.f95:58-86)
  for (int i = 0; i < Nh; i++) kx[i] = 2.0 * pi * (double)i / Lx;
  for (int j = 0; j < Ny; j++)
    ky[j] = (j < Ny / 2) ? 2.0 * pi * (double)j / Ly : 2.0 * pi * (double)(j - Ny) / Ly;
  // dsqrt(kx*kx + ky*ky) .ge. (dfloat(Nx+Ny)/2.0)/3.0 + 0     (src/derive2coh.f95:212)
  // The test is monotone in kx on every row, so row j is dealiased from
  // index cut[j] on.
  const double thr = ((double)(Nx + Ny) / 2.0) / 3.0 + 0;
  for (int j = 0; j < Ny; j++) {
    int c = Nh;
    for (int i = 0; i < Nh; i++) {
      volatile double a = kx[i] * kx[i];
      volatile double b = ky[j] * ky[j];
      volatile double s = a + b;
      if (std::sqrt((double)s) >= thr) { c = i; break; }
    }
    cut[j] = c;
  }
}

template <class T>
int Grid<T>::init(int nx, int ny, double lx, double ly, double pi_, cudaStream_t st) {
  if (!supported_length(nx) || !supported_length(ny)) {
    set_error("grid size not supported: Nx=" + std::to_string(nx) + " Ny=" + std::to_string(ny));
    return TARA_EUNSUPPORTED;
  }
  Nx = nx; Ny = ny; Nh = nx / 2 + 1;
  const int align = 128 / (int)sizeof(Cx<T>);
  ld = (Nh + align - 1) / align * align;
  Lx = lx; Ly = ly; pi = pi_;
  const int M = nx / 2;
  std::vector<Cx<T>> twc(ny), twr(M), twre(M + 1);
  for (int m = 0; m < ny; m++) { long double c, s; twiddle(m, ny, c, s); twc[m] = cx<T>((T)c, (T)s); }
  for (int m = 0; m < M; m++) { long double c, s; twiddle(m, M, c, s); twr[m] = cx<T>((T)c, (T)s); }
  for (int m = 0; m <= M; m++) { long double c, s; twiddle(m, nx, c, s); twre[m] = cx<T>((T)c, (T)s); }
  std::vector<double> kxd, kyd;
  std::vector<int> cut;
  wavenumbers(nx, ny, lx, ly, pi_, kxd, kyd, cut);
  std::vector<T> kx(kxd.begin(), kxd.end()), ky(kyd.begin(), kyd.end());
  auto al = [](size_t b) { return (b + 255) / 256 * 256; };
  size_t o_twc = 0, o_twr = o_twc + al(twc.size() * sizeof(Cx<T>)),
         o_twre = o_twr + al(twr.size() * sizeof(Cx<T>)),
         o_kx = o_twre + al(twre.size() * sizeof(Cx<T>)), o_ky = o_kx + al(kx.size() * sizeof(T)),
         o_cut = o_ky + al(ky.size() * sizeof(T)), o_status = o_cut + al(cut.size() * sizeof(int)),
         total = o_status + 256;
  if (cudaMalloc(&dmem, total) != cudaSuccess) {
    dmem = nullptr;
    set_error("cudaMalloc of grid tables failed");
    return TARA_ENOMEM;
  }
  char* b = (char*)dmem;
  std::vector<char> h(total, 0);
  std::memcpy(h.data() + o_twc, twc.data(), twc.size() * sizeof(Cx<T>));
  std::memcpy(h.data() + o_twr, twr.data(), twr.size() * sizeof(Cx<T>));
  std::memcpy(h.data() + o_twre, twre.data(), twre.size() * sizeof(Cx<T>));
  std::memcpy(h.data() + o_kx, kx.data(), kx.size() * sizeof(T));
  std::memcpy(h.data() + o_ky, ky.data(), ky.size() * sizeof(T));
  std::memcpy(h.data() + o_cut, cut.data(), cut.size() * sizeof(int));
  TARA_CUDA_TRY(cudaMemcpyAsync(b, h.data(), total, cudaMemcpyHostToDevice, st));
  TARA_CUDA_TRY(cudaStreamSynchronize(st));
  tb.tw_col = (const Cx<T>*)(b + o_twc);
  tb.tw_row = (const Cx<T>*)(b + o_twr);
  tb.tw_real = (const Cx<T>*)(b + o_twre);
  tb.kx = (const T*)(b + o_kx);
  tb.ky = (const T*)(b + o_ky);
  tb.cut = (const int*)(b + o_cut);
  tb.status = (int*)(b + o_status);
  int dev = 0, sms = 0;
  TARA_CUDA_TRY(cudaGetDevice(&dev));
  TARA_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  tb.sm_count = sms;
  tb.no_tma = 0;
  tb.wait_ns = 1000000000ull;
  tb.Nx = nx; tb.Ny = ny; tb.Nh = Nh; tb.ld = ld;
  double nn = (double)nx * (double)ny;
  tb.nn = (T)nn;
  tb.inv_nn = (T)(1.0 / nn);
  long long inn = (long long)nx * ny;
  tb.nn_pow2 = (inn & (inn - 1)) == 0;
  return TARA_OK;
}

static PFN_cuTensorMapEncodeTiled_v12000 tma_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  if (!fn) set_error("cuTensorMapEncodeTiled is not available from the driver");
  return fn;
}

int tma_encode_tile3(CUtensorMap* map, CUtensorMapDataType dt, void* base, uint64_t inner_elems, uint64_t rows,
                     uint64_t nf, uint64_t row_bytes, uint64_t field_bytes, uint32_t box_inner, uint32_t box_rows) {
  auto fn = tma_encoder();
  if (!fn) return TARA_ECUDA;
  cuuint64_t dims[3] = {inner_elems, rows, nf};
  cuuint64_t strides[2] = {row_bytes, field_bytes};
  cuuint32_t box[3] = {box_inner, box_rows, 1};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = fn(map, dt, 3, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled (3D) failed with CUresult " + std::to_string((int)r));
    return TARA_ECUDA;
  }
  return TARA_OK;
}

int tma_encode_tile(CUtensorMap* map, CUtensorMapDataType dt, void* base, uint64_t inner_elems, uint64_t rows,
                    uint64_t row_bytes, uint32_t box_inner, uint32_t box_rows) {
  auto fn = tma_encoder();
  if (!fn) return TARA_ECUDA;
  cuuint64_t dims[2] = {inner_elems, rows};
  cuuint64_t strides[1] = {row_bytes};
  cuuint32_t box[2] = {box_inner, box_rows};
  cuuint32_t es[2] = {1, 1};
  CUresult r = fn(map, dt, 2, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed with CUresult " + std::to_string((int)r));
    return TARA_ECUDA;
  }
  return TARA_OK;
}

template <class T>
void Grid<T>::release() {
  if (dmem) cudaFree(dmem);
  dmem = nullptr;
}

template <class T>
int FieldPool<T>::alloc(const Grid<T>& g, int n, cudaStream_t st) {
  elems = g.field_elems();
  count = n;
  size_t bytes = elems * sizeof(Cx<T>) * (size_t)n;
  if (cudaMalloc(&base, bytes) != cudaSuccess) {
    base = nullptr;
    set_error("cudaMalloc of " + std::to_string(bytes) + " bytes of field storage failed");
    return TARA_ENOMEM;
  }
  TARA_CUDA_TRY(cudaMemsetAsync(base, 0, bytes, st));
  return TARA_OK;
}
template <class T>
void FieldPool<T>::release() {
  if (base) cudaFree(base);
  base = nullptr;
}

template struct Grid<double>;
template struct Grid<float>;
template struct FieldPool<double>;
template struct FieldPool<float>;

}  // namespace tara
