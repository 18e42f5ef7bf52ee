// Binary checkpoint / restart of a session: the state, the AB2/Euler history
// (the previous derivative), the model, grid and parameters, and the
// caller's step count and time.  The reference has no restart; its drivers
// always start from an initial condition (src/main2com.f95:215-343,
// src/main2coh.f95:176-257), so the format is this library's own.
//
// File layout (little-endian, 8-byte aligned throughout):
//   header, 192 bytes:
//     char   magic[8] = "TARA2DCK"
//     uint32 version = 1
//     int32  model, precision, Nx, Ny, nf, fix_curlB
//     int32  flags (bit 0: history present)
//     int64  step
//     double time
//     double params[17]: Lx, Ly, pi, dt, mux, muy, ms, CS, spheat, mu,
//                        mu_0, eta, kf, A, nu, alpha, lambda
//   nf state fields, then (flags bit 0) nf history fields, each the
//     [Ny][Nh] complex array of the host API (re, im as FP64) whatever the
//     session's precision
//   checksum, 16 bytes: uint64 s1 = sum of every preceding 8-byte word w_i,
//     uint64 s2 = sum of (i + 1) * w_i, both modulo 2^64
// The file is written under path + ".tmp" and renamed over path once
// complete, so an interrupted write leaves an earlier checkpoint intact.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "plan.h"
#include "session.h"

namespace {

constexpr char kMagic[8] = {'T', 'A', 'R', 'A', '2', 'D', 'C', 'K'};
constexpr uint32_t kVersion = 1;
constexpr int kParams = 17;
constexpr size_t kHeaderBytes = 192;

struct Header {
  uint32_t version;
  int32_t model, precision, Nx, Ny, nf, fix_curlB, flags;
  int64_t step;
  double time;
  double prm[kParams];
};

void params_to(const tara_params& p, double* v) {
  const double a[kParams] = {p.Lx, p.Ly,   p.pi, p.dt, p.mux, p.muy, p.ms, p.CS,  p.spheat,
                             p.mu, p.mu_0, p.eta, p.kf, p.A,  p.nu,  p.alpha, p.lambda};
  std::memcpy(v, a, sizeof(a));
}
void params_from(const double* v, tara_params& p) {
  double* a[kParams] = {&p.Lx, &p.Ly,   &p.pi, &p.dt, &p.mux, &p.muy, &p.ms, &p.CS,  &p.spheat,
                        &p.mu, &p.mu_0, &p.eta, &p.kf, &p.A,  &p.nu,  &p.alpha, &p.lambda};
  for (int k = 0; k < kParams; k++) *a[k] = v[k];
}

void put(std::vector<unsigned char>& b, const void* p, size_t n) {
  const unsigned char* c = static_cast<const unsigned char*>(p);
  b.insert(b.end(), c, c + n);
}

std::vector<unsigned char> encode_header(const Header& h) {
  std::vector<unsigned char> b;
  put(b, kMagic, 8);
  put(b, &h.version, 4);
  const int32_t ints[7] = {h.model, h.precision, h.Nx, h.Ny, h.nf, h.fix_curlB, h.flags};
  put(b, ints, sizeof(ints));
  put(b, &h.step, 8);
  put(b, &h.time, 8);
  put(b, h.prm, sizeof(h.prm));
  return b;  // 8 + 4 + 28 + 8 + 8 + 136 = 192 bytes
}

bool decode_header(const unsigned char* b, Header& h) {
  if (std::memcmp(b, kMagic, 8) != 0) return false;
  std::memcpy(&h.version, b + 8, 4);
  int32_t ints[7];
  std::memcpy(ints, b + 12, sizeof(ints));
  h.model = ints[0]; h.precision = ints[1]; h.Nx = ints[2]; h.Ny = ints[3];
  h.nf = ints[4]; h.fix_curlB = ints[5]; h.flags = ints[6];
  std::memcpy(&h.step, b + 40, 8);
  std::memcpy(&h.time, b + 48, 8);
  std::memcpy(h.prm, b + 56, sizeof(h.prm));
  return true;
}

// running (s1, s2) over 8-byte words; `index` counts the words seen so far
struct Checksum {
  uint64_t s1 = 0, s2 = 0, index = 0;
  void add(const void* p, size_t n) {  // n is a multiple of 8
    const unsigned char* c = static_cast<const unsigned char*>(p);
    for (size_t k = 0; k < n; k += 8) {
      uint64_t w;
      std::memcpy(&w, c + k, 8);
      index++;
      s1 += w;
      s2 += index * w;
    }
  }
};

bool write_all(FILE* f, const void* p, size_t n, Checksum* cs) {
  if (cs) cs->add(p, n);
  return std::fwrite(p, 1, n, f) == n;
}
bool read_all(FILE* f, void* p, size_t n, Checksum* cs) {
  if (std::fread(p, 1, n, f) != n) return false;
  if (cs) cs->add(p, n);
  return true;
}

}  // namespace

extern "C" int tara_checkpoint_write(tara_session* s, const char* path, long long step, double time) {
  using tara::set_error;
  if (!s || !path) return TARA_EINVAL;
  const size_t nh = (size_t)(s->Nx / 2 + 1), per = nh * (size_t)s->Ny * 2;  // doubles per field
  std::vector<double> buf(2 * (size_t)s->nf * per);
  double* fp[12];
  for (int q = 0; q < 2 * s->nf; q++) fp[q] = buf.data() + q * per;
  int r = s->get_fields(0, fp);
  if (r == TARA_OK) r = s->get_fields(1, fp + s->nf);
  if (r != TARA_OK) return s->fail_if(r);
  Header h{};
  h.version = kVersion;
  h.model = s->model; h.precision = s->precision; h.Nx = s->Nx; h.Ny = s->Ny; h.nf = s->nf;
  h.fix_curlB = s->p.fix_curlB;
  h.flags = 1;
  h.step = step;
  h.time = time;
  params_to(s->p, h.prm);
  const std::vector<unsigned char> hb = encode_header(h);
  if (hb.size() != kHeaderBytes) { set_error("checkpoint header size"); return TARA_EINVAL; }
  const std::string tmp = std::string(path) + ".tmp";
  FILE* f = std::fopen(tmp.c_str(), "wb");
  if (!f) { set_error("cannot open " + tmp); return TARA_EINVAL; }
  Checksum cs;
  bool ok = write_all(f, hb.data(), hb.size(), &cs) && write_all(f, buf.data(), buf.size() * 8, &cs);
  const uint64_t tail[2] = {cs.s1, cs.s2};
  ok = ok && write_all(f, tail, sizeof(tail), nullptr);
  ok = (std::fclose(f) == 0) && ok;
  if (!ok || std::rename(tmp.c_str(), path) != 0) {
    std::remove(tmp.c_str());
    set_error(std::string("write of checkpoint ") + path + " failed");
    return TARA_EINVAL;
  }
  return TARA_OK;
}

extern "C" int tara_checkpoint_read(tara_session* s, const char* path, long long* step, double* time) {
  using tara::set_error;
  if (!s || !path) return TARA_EINVAL;
  FILE* f = std::fopen(path, "rb");
  if (!f) { set_error(std::string("cannot open ") + path); return TARA_EINVAL; }
  auto fail = [&](const std::string& why) {
    std::fclose(f);
    set_error(std::string("checkpoint ") + path + ": " + why);
    return TARA_EINVAL;
  };
  unsigned char hb[kHeaderBytes];
  Checksum cs;
  Header h{};
  if (!read_all(f, hb, kHeaderBytes, &cs) || !decode_header(hb, h)) return fail("not a checkpoint file");
  if (h.version != kVersion) return fail("unsupported version " + std::to_string(h.version));
  if (h.model != s->model || h.Nx != s->Nx || h.Ny != s->Ny || h.nf != s->nf)
    return fail("model or grid differs from the session's");
  const bool hist = (h.flags & 1) != 0;
  const size_t nh = (size_t)(s->Nx / 2 + 1), per = nh * (size_t)s->Ny * 2;
  std::vector<double> buf((hist ? 2 : 1) * (size_t)s->nf * per);
  if (!read_all(f, buf.data(), buf.size() * 8, &cs)) return fail("truncated");
  uint64_t tail[2];
  if (!read_all(f, tail, sizeof(tail), nullptr)) return fail("truncated");
  if (tail[0] != cs.s1 || tail[1] != cs.s2) return fail("checksum mismatch");
  std::fclose(f);
  tara_params p = s->p;
  params_from(h.prm, p);
  p.fix_curlB = h.fix_curlB;
  s->p = p;
  TARA_TRY(s->fail_if(s->apply_params()));
  double* fp[12];
  for (int q = 0; q < (hist ? 2 : 1) * s->nf; q++) fp[q] = buf.data() + q * per;
  TARA_TRY(s->fail_if(s->set_fields(0, fp)));
  if (hist) TARA_TRY(s->fail_if(s->set_fields(1, fp + s->nf)));
  if (step) *step = h.step;
  if (time) *time = h.time;
  return TARA_OK;
}
