// Shared-memory Stockham FFT building blocks for the pseudo-spectral path.
//
// Everything here is __host__ __device__ so that the same index arithmetic
// runs in a host-side simulation (tests/cpu_sim) and in the sm_100a kernels.
//
// Conventions
//   * complex values are Cx<T> {x = re, y = im}; T is double or float.
//   * DIR = -1 : forward  X[k] = sum_n x[n] e^{-2 pi i nk/L}
//     DIR = +1 : inverse  x[n] = sum_k X[k] e^{+2 pi i nk/L}   (unnormalised)
//   * A length-L transform is split into stages with radices R_0..R_{S-1}
//     (RadixPlan<L>).  Every thread owns P complex values; at stage s it runs
//     P/R_s butterflies of radix R_s.  Stage s (Stockham autosort, Ns = R_0..R_{s-1}):
//         in[r]  = data[j + r*L/R]                 r = 0..R-1
//         in[r] *= w^( (j mod Ns) * r * L/(Ns*R) ) (w = e^{DIR 2 pi i/L})
//         DFT_R(in)
//         data'[(j/Ns)*Ns*R + (j mod Ns) + r*Ns] = in[r]
//     which leaves the output in natural order after the last stage.
#pragma once
#include <stdint.h>

#ifndef TARA_HD
#if defined(__CUDACC__)
#define TARA_HD __host__ __device__ __forceinline__
#else
#define TARA_HD inline
#endif
#endif
#ifndef TARA_HDC
#if defined(__CUDACC__)
#define TARA_HDC __host__ __device__
#else
#define TARA_HDC
#endif
#endif

namespace tara {

// Aligned to its size so that shared/global accesses are single 16-byte
// (double) or 8-byte (float) transactions.
template <class T>
struct alignas(2 * sizeof(T)) Cx {
  T x, y;
};

template <class T> TARA_HD Cx<T> cx(T a, T b) { Cx<T> r; r.x = a; r.y = b; return r; }
template <class T> TARA_HD Cx<T> operator+(Cx<T> a, Cx<T> b) { return cx<T>(a.x + b.x, a.y + b.y); }
template <class T> TARA_HD Cx<T> operator-(Cx<T> a, Cx<T> b) { return cx<T>(a.x - b.x, a.y - b.y); }
template <class T> TARA_HD Cx<T> operator-(Cx<T> a) { return cx<T>(-a.x, -a.y); }
template <class T> TARA_HD Cx<T> cmul(Cx<T> a, Cx<T> b) {
  return cx<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <class T> TARA_HD Cx<T> conj(Cx<T> a) { return cx<T>(a.x, -a.y); }
template <class T> TARA_HD Cx<T> rmul(T r, Cx<T> a) { return cx<T>(r * a.x, r * a.y); }
// (0,1)*k*z with Fortran complex-multiply rules: (0*a - k*b, 0*b + k*a) == (-k*b, k*a)
template <class T> TARA_HD Cx<T> ikmul(T k, Cx<T> a) { return cx<T>(-(k * a.y), k * a.x); }
// multiply by DIR*i  (DIR = +1 : i,  DIR = -1 : -i)
template <int DIR, class T> TARA_HD Cx<T> mul_i(Cx<T> a) {
  return DIR > 0 ? cx<T>(-a.y, a.x) : cx<T>(a.y, -a.x);
}
// multiply by e^{DIR*2*pi*i*m/16} for compile-time m (m in 0..15)
template <int DIR, int M, class T> TARA_HD Cx<T> w16(Cx<T> a) {
  constexpr int m = M & 15;
  const T c1 = (T)0.92387953251128675613L;  // cos(pi/8)
  const T s1 = (T)0.38268343236508977173L;  // sin(pi/8)
  const T h = (T)0.70710678118654752440L;   // sqrt(1/2)
  // e^{i theta}, theta = 2 pi m/16, as (c, s); DIR flips s
  if constexpr (m == 0) return a;
  else if constexpr (m == 4) return mul_i<DIR>(a);
  else if constexpr (m == 8) return -a;
  else if constexpr (m == 12) return mul_i<-DIR>(a);
  else {
    T c, s;
    if constexpr (m == 1) { c = c1; s = s1; }
    else if constexpr (m == 2) { c = h; s = h; }
    else if constexpr (m == 3) { c = s1; s = c1; }
    else if constexpr (m == 5) { c = -s1; s = c1; }
    else if constexpr (m == 6) { c = -h; s = h; }
    else if constexpr (m == 7) { c = -c1; s = s1; }
    else if constexpr (m == 9) { c = -c1; s = -s1; }
    else if constexpr (m == 10) { c = -h; s = -h; }
    else if constexpr (m == 11) { c = -s1; s = -c1; }
    else if constexpr (m == 13) { c = s1; s = -c1; }
    else if constexpr (m == 14) { c = h; s = -h; }
    else { c = c1; s = -s1; }
    if (DIR < 0) s = -s;
    return cx<T>(a.x * c - a.y * s, a.x * s + a.y * c);
  }
}

// ---------------------------------------------------------------- radix DFTs
// In-place DFT of v[0..R-1] with stride ST (the values are v[0], v[ST], ...),
// natural-order output.
template <int DIR, class T, int ST = 1> TARA_HD void dft2(Cx<T>* v) {
  Cx<T> a = v[0], b = v[ST];
  v[0] = a + b;
  v[ST] = a - b;
}
template <int DIR, class T, int ST = 1> TARA_HD void dft4(Cx<T>* v) {
  Cx<T> a0 = v[0] + v[2 * ST], a1 = v[0] - v[2 * ST];
  Cx<T> b0 = v[ST] + v[3 * ST], b1 = mul_i<DIR>(v[ST] - v[3 * ST]);
  v[0] = a0 + b0;
  v[2 * ST] = a0 - b0;
  v[ST] = a1 + b1;
  v[3 * ST] = a1 - b1;
}
template <int DIR, class T> TARA_HD void dft8(Cx<T>* v) {
  // radix-2 x 4: E = DFT4(even), O = DFT4(odd), X[k] = E[k] + W8^k O[k]
  Cx<T> e[4] = {v[0], v[2], v[4], v[6]};
  Cx<T> o[4] = {v[1], v[3], v[5], v[7]};
  dft4<DIR>(e);
  dft4<DIR>(o);
  o[1] = w16<DIR, 2>(o[1]);
  o[2] = w16<DIR, 4>(o[2]);
  o[3] = w16<DIR, 6>(o[3]);
#pragma unroll
  for (int k = 0; k < 4; k++) {
    v[k] = e[k] + o[k];
    v[k + 4] = e[k] - o[k];
  }
}
template <int DIR, class T> TARA_HD void dft16(Cx<T>* v) {
  // 4 x 4: X[k1 + 4 k2] = sum_n2 W4^{n2 k2} W16^{n2 k1} sum_n1 x[4 n1 + n2] W4^{n1 k1}
  Cx<T> y[16];
#pragma unroll
  for (int n2 = 0; n2 < 4; n2++) {
    Cx<T> t[4] = {v[n2], v[4 + n2], v[8 + n2], v[12 + n2]};
    dft4<DIR>(t);
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) y[4 * n2 + k1] = t[k1];
  }
  // twiddles W16^{n2*k1}
  y[5] = w16<DIR, 1>(y[5]);
  y[6] = w16<DIR, 2>(y[6]);
  y[7] = w16<DIR, 3>(y[7]);
  y[9] = w16<DIR, 2>(y[9]);
  y[10] = w16<DIR, 4>(y[10]);
  y[11] = w16<DIR, 6>(y[11]);
  y[13] = w16<DIR, 3>(y[13]);
  y[14] = w16<DIR, 6>(y[14]);
  y[15] = w16<DIR, 9>(y[15]);
#pragma unroll
  for (int k1 = 0; k1 < 4; k1++) {
    Cx<T> t[4] = {y[k1], y[4 + k1], y[8 + k1], y[12 + k1]};
    dft4<DIR>(t);
#pragma unroll
    for (int k2 = 0; k2 < 4; k2++) v[k1 + 4 * k2] = t[k2];
  }
}
template <int DIR, class T> TARA_HD void dft3(Cx<T>* v) {
  const T c = (T)-0.5L;
  const T s = (T)0.86602540378443864676L * (T)DIR;  // DIR * sin(2 pi/3)
  Cx<T> a = v[0], b = v[1], d = v[2];
  Cx<T> t = b + d, u = b - d;
  v[0] = a + t;
  Cx<T> m = cx<T>(a.x + c * t.x, a.y + c * t.y);
  Cx<T> q = cx<T>(-s * u.y, s * u.x);  // i * s * u
  v[1] = m + q;
  v[2] = m - q;
}
template <int DIR, class T> TARA_HD void dft6(Cx<T>* v) {
  // 3 x 2 (Good-Thomas free): X[k] with n = 2 n1 + n2 ... use radix-2 of DFT3:
  // E = DFT3(v0,v2,v4), O = DFT3(v1,v3,v5), X[k] = E[k mod 3] + W6^k O[k mod 3]
  Cx<T> e[3] = {v[0], v[2], v[4]};
  Cx<T> o[3] = {v[1], v[3], v[5]};
  dft3<DIR>(e);
  dft3<DIR>(o);
  const T c = (T)0.5L, s = (T)0.86602540378443864676L * (T)DIR;
  // W6^1 = (1/2, DIR*sqrt3/2), W6^2 = (-1/2, DIR*sqrt3/2)
  Cx<T> o1 = cx<T>(o[1].x * c - o[1].y * s, o[1].x * s + o[1].y * c);
  Cx<T> o2 = cx<T>(-o[2].x * c - o[2].y * s, o[2].x * s - o[2].y * c);
  v[0] = e[0] + o[0];
  v[3] = e[0] - o[0];
  v[1] = e[1] + o1;
  v[4] = e[1] - o1;
  v[2] = e[2] + o2;
  v[5] = e[2] - o2;
}
template <int R, int DIR, class T> TARA_HD void dft(Cx<T>* v) {
  if constexpr (R == 2) dft2<DIR>(v);
  else if constexpr (R == 3) dft3<DIR>(v);
  else if constexpr (R == 4) dft4<DIR>(v);
  else if constexpr (R == 6) dft6<DIR>(v);
  else if constexpr (R == 8) dft8<DIR>(v);
  else if constexpr (R == 16) dft16<DIR>(v);
  else static_assert(R == 2, "unsupported radix");
}

// ---------------------------------------------------------------- radix plans
// RadixPlan<L, P>: a length-L transform whose threads own P complex values
// each; every radix divides P.  S = number of stages (<= 4).
template <int L, int P> struct RadixPlan;
#define TARA_PLAN(L_, P_, S_, R0, R1, R2, R3)                     \
  template <> struct RadixPlan<L_, P_> {                          \
    static constexpr int S = S_;                                  \
    static constexpr int R[4] = {R0, R1, R2, R3};                 \
  };
TARA_PLAN(8, 8, 1, 8, 1, 1, 1)
TARA_PLAN(16, 8, 2, 8, 2, 1, 1)
TARA_PLAN(32, 8, 2, 8, 4, 1, 1)
TARA_PLAN(64, 8, 2, 8, 8, 1, 1)
TARA_PLAN(128, 8, 3, 8, 8, 2, 1)
TARA_PLAN(256, 8, 3, 8, 8, 4, 1)
TARA_PLAN(512, 8, 3, 8, 8, 8, 1)
TARA_PLAN(1024, 8, 4, 8, 8, 8, 2)
TARA_PLAN(2048, 8, 4, 8, 8, 8, 4)
TARA_PLAN(4096, 8, 4, 8, 8, 8, 8)
TARA_PLAN(16, 16, 1, 16, 1, 1, 1)
TARA_PLAN(32, 16, 2, 16, 2, 1, 1)
TARA_PLAN(64, 16, 2, 16, 4, 1, 1)
TARA_PLAN(128, 16, 2, 16, 8, 1, 1)
TARA_PLAN(256, 16, 2, 16, 16, 1, 1)
TARA_PLAN(512, 16, 3, 16, 16, 2, 1)
TARA_PLAN(1024, 16, 3, 16, 16, 4, 1)
TARA_PLAN(2048, 16, 3, 16, 16, 8, 1)
TARA_PLAN(4096, 16, 3, 16, 16, 16, 1)
TARA_PLAN(48, 24, 3, 8, 2, 3, 1)
TARA_PLAN(96, 24, 3, 8, 4, 3, 1)
TARA_PLAN(192, 24, 3, 8, 8, 3, 1)
TARA_PLAN(384, 24, 3, 8, 8, 6, 1)
TARA_PLAN(768, 24, 4, 8, 8, 6, 2)
#undef TARA_PLAN

// Ns of stage s: product of the radices of the stages before it
template <int L, int P> TARA_HDC constexpr int stage_ns(int s) {
  int ns = 1;
  for (int i = 0; i < s; i++) ns *= RadixPlan<L, P>::R[i];
  return ns;
}

// A batch of B transforms of length L owned by NT threads, P values each.
// Butterfly b of stage s:  t = b % B (transform), j = b / B (butterfly within the transform).
// Thread `tid` owns butterflies b = tid + q*NT, q = 0..P/R_s-1.
template <int L, int B, int P_> struct BatchFFT {
  using Pl = RadixPlan<L, P_>;
  static constexpr int P = P_;
  static constexpr int S = Pl::S;
  static constexpr int NT = B * L / P;
  static_assert(B * L % P == 0, "batch does not split into whole threads");

  // element index (t, i) of input value r of butterfly q (thread tid) at stage s
  template <int s>
  TARA_HD static constexpr void in_pos(int tid, int q, int r, int& t, int& i) {
    constexpr int R = Pl::R[s];
    int b = tid + q * NT;
    t = b % B;
    int j = b / B;
    i = j + r * (L / R);
  }
  template <int s>
  TARA_HD static constexpr void out_pos(int tid, int q, int r, int& t, int& i) {
    constexpr int R = Pl::R[s];
    constexpr int Ns = stage_ns<L, P_>(s);
    int b = tid + q * NT;
    t = b % B;
    int j = b / B;
    i = (j / Ns) * Ns * R + (j % Ns) + r * Ns;
  }
  // True when the exchange in front of stage s (s >= 1) is a swap between
  // threads tid and tid ^ 16 of 32: one transform (B = 1) on 32 threads whose
  // stage s is radix 2, and every input of stage s either already sits in its
  // thread's slot 2q + hb or sits in the partner's slot 2q + hb (hb = bit 4
  // of tid), checked against in_pos/out_pos for every thread and slot.  Holds
  // for the 512-point transforms with 16 values per thread (stages 16, 16, 2).
  template <int s>
  TARA_HDC static constexpr bool halves_exchange() {
    if (B != 1 || NT != 32 || Pl::R[s] != 2) return false;
    constexpr int Rp = Pl::R[s - 1];
    for (int tid = 0; tid < 32; tid++) {
      const int hb = (tid >> 4) & 1;
      for (int q = 0; q < P / 2; q++)
        for (int r = 0; r < 2; r++) {
          int t = 0, i = 0, ts = 0, is = 0;
          in_pos<s>(tid, q, r, t, i);
          const int src = r == hb ? tid : tid ^ 16, slot = 2 * q + hb;
          out_pos<s - 1>(src, slot / Rp, slot % Rp, ts, is);
          if (is != i) return false;
        }
    }
    return true;
  }
  // twiddle + butterflies of stage s on v[P] (v[q*R + r] = input r of butterfly q).
  // tw[m] = e^{-2 pi i m / L} (forward table); DIR selects the conjugate.
  template <int s, int DIR, class T, class TW>
  TARA_HD static void compute(int tid, Cx<T>* v, const TW& tw) {
    constexpr int R = Pl::R[s];
    constexpr int Ns = stage_ns<L, P_>(s);
    constexpr int Q = P / R;
#pragma unroll
    for (int q = 0; q < Q; q++) {
      Cx<T>* u = v + q * R;
      if constexpr (Ns > 1) {
        int b = tid + q * NT;
        int j = b / B;
        int jm = j % Ns;
        constexpr int stride = L / (Ns * R);
        // w^r for r = 1..R-1 from the table entries w^1, w^2, w^4, w^8 (at
        // most two further products each, so within a few ulp of the table),
        // applied as soon as each is formed to keep few of them live
        const int m1 = jm * stride;
        auto apply = [&](int r, Cx<T> wr) {
          if (DIR > 0) wr.y = -wr.y;
          u[r] = cmul(u[r], wr);
        };
        const Cx<T> w1 = tw(m1);
        Cx<T> w8;
        if constexpr (R >= 16) {
          w8 = tw(8 * m1);
          apply(8, w8);
          apply(9, cmul(w8, w1));
        }
        apply(1, w1);
        if constexpr (R >= 3) {
          const Cx<T> w2 = tw(2 * m1);
          apply(2, w2);
          if constexpr (R >= 16) apply(10, cmul(w8, w2));
          if constexpr (R >= 4) {
            const Cx<T> w3 = cmul(w2, w1);
            apply(3, w3);
            if constexpr (R >= 16) apply(11, cmul(w8, w3));
            if constexpr (R >= 5) {
              const Cx<T> w4 = tw(4 * m1);
              apply(4, w4);
              if constexpr (R >= 16) apply(12, cmul(w8, w4));
              if constexpr (R >= 6) {
                const Cx<T> w5 = cmul(w4, w1);
                apply(5, w5);
                if constexpr (R >= 16) apply(13, cmul(w8, w5));
              }
              if constexpr (R >= 8) {
                const Cx<T> w6 = cmul(w4, w2);
                apply(6, w6);
                const Cx<T> w7 = cmul(w4, w3);
                apply(7, w7);
                if constexpr (R >= 16) {
                  apply(14, cmul(w8, w6));
                  apply(15, cmul(w8, w7));
                }
              }
            }
          }
        }
      }
      dft<R, DIR>(u);
    }
  }
};

}  // namespace tara
