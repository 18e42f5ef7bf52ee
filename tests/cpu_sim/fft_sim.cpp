// Host simulation of the Stockham engine in tara2d_b200/csrc/fft_core.cuh.
// Runs the per-thread stage code for every thread of a batch in turn (one
// pass per barrier interval) and checks the result against a direct DFT in
// long double.  Built and run by tests/test_fft_engine_cpu.py.
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "../../tara2d_b200/csrc/fft_core.cuh"

using namespace tara;

template <int L>
struct Table {
  std::vector<Cx<double>> w;
  Table() : w(L) {
    for (int m = 0; m < L; m++) {
      long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)L;
      w[m] = cx<double>((double)cosl(a), (double)sinl(a));
    }
  }
  Cx<double> operator()(int m) const { return w[m]; }
};

template <int L, int B, int P, int DIR, int s>
void run_stage_load(const std::vector<Cx<double>>& data, std::vector<std::vector<Cx<double>>>& regs) {
  using F = BatchFFT<L, B, P>;
  constexpr int R = F::Pl::R[s];
  for (int tid = 0; tid < F::NT; tid++)
    for (int q = 0; q < P / R; q++)
      for (int r = 0; r < R; r++) {
        int t, i;
        F::template in_pos<s>(tid, q, r, t, i);
        regs[tid][q * R + r] = data[i * B + t];
      }
}
template <int L, int B, int P, int DIR, int s>
void run_stage_store(std::vector<Cx<double>>& data, const std::vector<std::vector<Cx<double>>>& regs) {
  using F = BatchFFT<L, B, P>;
  constexpr int R = F::Pl::R[s];
  for (int tid = 0; tid < F::NT; tid++)
    for (int q = 0; q < P / R; q++)
      for (int r = 0; r < R; r++) {
        int t, i;
        F::template out_pos<s>(tid, q, r, t, i);
        data[i * B + t] = regs[tid][q * R + r];
      }
}
// The register exchange of the row kernels (spectral.cuh, warp_halves_swap):
// thread tid keeps slot 2q + hb and takes slot 2q + 1 - hb from thread
// tid ^ 16, as __shfl_xor_sync(.., 16) does within a warp.
template <int L, int B, int P>
void run_halves_swap(std::vector<std::vector<Cx<double>>>& regs) {
  std::vector<std::vector<Cx<double>>> old = regs;
  for (int tid = 0; tid < 32; tid++) {
    const int hb = (tid >> 4) & 1;
    for (int q = 0; q < P / 2; q++) regs[tid][2 * q + 1 - hb] = old[tid ^ 16][2 * q + hb];
  }
}
// Stage s: its inputs from the previous stage's registers (through the
// exchange buffer, or by the lane swap where BatchFFT::halves_exchange
// holds, as the device code chooses), butterflies; the last stage's outputs
// are stored.
template <int L, int B, int P, int DIR, int s>
void run_stages(std::vector<Cx<double>>& data, std::vector<std::vector<Cx<double>>>& regs, const Table<L>& tw,
                int& swaps) {
  using F = BatchFFT<L, B, P>;
  if constexpr (s < F::S) {
    if constexpr (s == 0) {
      run_stage_load<L, B, P, DIR, 0>(data, regs);
    } else if constexpr (F::template halves_exchange<s>()) {
      run_halves_swap<L, B, P>(regs);
      swaps++;
    } else {
      run_stage_store<L, B, P, DIR, s - 1>(data, regs);
      run_stage_load<L, B, P, DIR, s>(data, regs);
    }
    for (int tid = 0; tid < F::NT; tid++) F::template compute<s, DIR>(tid, regs[tid].data(), tw);
    if constexpr (s == F::S - 1) run_stage_store<L, B, P, DIR, s>(data, regs);
    run_stages<L, B, P, DIR, s + 1>(data, regs, tw, swaps);
  }
}

template <int L, int B, int P, int DIR>
int check() {
  using F = BatchFFT<L, B, P>;
  std::vector<Cx<double>> data(L * B), orig;
  srand(L * 131 + B * 7 + P + (DIR > 0));
  for (auto& v : data) v = cx<double>(rand() / (double)RAND_MAX - 0.5, rand() / (double)RAND_MAX - 0.5);
  orig = data;
  std::vector<std::vector<Cx<double>>> regs(F::NT, std::vector<Cx<double>>(P));
  Table<L> tw;
  int swaps = 0;
  run_stages<L, B, P, DIR, 0>(data, regs, tw, swaps);
  double maxerr = 0, maxv = 0;
  for (int t = 0; t < B; t++)
    for (int k = 0; k < L; k++) {
      std::complex<long double> acc = 0;
      for (int n = 0; n < L; n++) {
        long double a = DIR * 2.0L * 3.14159265358979323846264338327950288L * (long double)((long long)n * k % L) / L;
        acc += std::complex<long double>(orig[n * B + t].x, orig[n * B + t].y) * std::complex<long double>(cosl(a), sinl(a));
      }
      double ex = (double)std::abs(acc - std::complex<long double>(data[k * B + t].x, data[k * B + t].y));
      maxerr = std::fmax(maxerr, ex);
      maxv = std::fmax(maxv, (double)std::abs(acc));
    }
  double rel = maxerr / maxv;
  bool ok = rel < 1e-14;
  printf("L=%5d B=%d P=%2d DIR=%+d threads=%4d lane_swaps=%d rel_err=%.3e %s\n", L, B, P, DIR, F::NT, swaps, rel,
         ok ? "ok" : "FAIL");
  return ok ? 0 : 1;
}

#define BOTH(L, B, P) fails += check<L, B, P, -1>() + check<L, B, P, +1>();
int main() {
  int fails = 0;
  BOTH(8, 1, 8) BOTH(16, 1, 8) BOTH(32, 2, 8) BOTH(64, 1, 8) BOTH(128, 2, 8) BOTH(256, 1, 8)
  BOTH(512, 1, 8) BOTH(1024, 1, 8) BOTH(2048, 1, 8)
  BOTH(16, 4, 16) BOTH(32, 1, 16) BOTH(64, 8, 16) BOTH(128, 8, 16) BOTH(256, 4, 16) BOTH(512, 4, 16) BOTH(512, 1, 16)
  BOTH(1024, 4, 16) BOTH(2048, 2, 16) BOTH(4096, 1, 16)
  BOTH(48, 2, 24) BOTH(96, 1, 24) BOTH(192, 1, 24) BOTH(384, 4, 24) BOTH(768, 1, 24)
  // the column tiles the MHD column-forward pass runs (kx columns x values per thread)
  BOTH(256, 8, 16) BOTH(512, 2, 8) BOTH(512, 4, 8) BOTH(1024, 4, 8) BOTH(2048, 2, 8) BOTH(2048, 4, 8)
  BOTH(4096, 2, 8) BOTH(4096, 2, 16)
  printf("%s\n", fails ? "FAILED" : "ALL OK");
  return fails ? 1 : 0;
}
