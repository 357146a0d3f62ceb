// Four-step transforms with register-resident DFT codelets (sm_100a).
//
// A line of length N = N1 N2 (both at most 32) is transformed in two passes:
//   pass 1, item t < N2:  v[m] = x[t + N2 m] (m < N1); N1-point DFT over m; v[k2] *= w^(t k2),
//                         w = e^{sign 2 pi i / N}; written back to positions t + N2 k2
//                         (the positions it read, so the pass runs in place);
//   pass 2, item k2 < N1: v[t] = y[t + N2 k2] (t < N2); N2-point DFT over t;
//                         X[k2 + N1 k1] = v[k1].
// Each point is read and written once per pass; the DFTs run in registers with
// compile-time twiddles, and only the pass-1 twiddles w^(t k2) come from a table
// (e^{-2 pi i t/N}, double-evaluated on the host, rounded to float).
//
// The codelets of fft_core.cuh cover radices 2..9 and 16; the others used here are
// composites R = A B (Cooley-Tukey in registers) whose twiddles cos/sin(2 pi m / R) are
// computed at compile time from their Taylor series in double.
#pragma once
#include "fft_core.cuh"

namespace crava {

// ------------------------------------------------------------------ compile-time trig

constexpr double kTwoPi = 6.283185307179586476925286766559;

// Taylor series of sin / cos, |x| <= pi/4: 12 terms are exact to double rounding.
constexpr double ct_sin_series(double x) {
  double term = x, sum = x;
  for (int k = 1; k < 12; k++) {
    term *= -x * x / ((2.0 * k) * (2.0 * k + 1.0));
    sum += term;
  }
  return sum;
}
constexpr double ct_cos_series(double x) {
  double term = 1.0, sum = 1.0;
  for (int k = 1; k < 12; k++) {
    term *= -x * x / ((2.0 * k - 1.0) * (2.0 * k));
    sum += term;
  }
  return sum;
}
// cos and sin of 2 pi m / R with the reduction done on the integers: 8 m / R falls in an
// octant o, and the residual angle is at most pi/4.
constexpr double ct_cos2pi(int m, int R) {
  m = ((m % R) + R) % R;
  // angle = 2 pi m / R = (pi / 4) (8 m / R); nearest multiple of pi/2: q = round(4 m / R)
  const int q = (8 * m + R) / (2 * R);                 // 0..4
  const double r = kTwoPi * ((double)m / R) - (kTwoPi / 4.0) * q;   // |r| <= pi/4
  switch (q & 3) {
    case 0: return ct_cos_series(r);
    case 1: return -ct_sin_series(r);
    case 2: return -ct_cos_series(r);
    default: return ct_sin_series(r);
  }
}
constexpr double ct_sin2pi(int m, int R) {
  m = ((m % R) + R) % R;
  const int q = (8 * m + R) / (2 * R);
  const double r = kTwoPi * ((double)m / R) - (kTwoPi / 4.0) * q;
  switch (q & 3) {
    case 0: return ct_sin_series(r);
    case 1: return ct_cos_series(r);
    case 2: return -ct_sin_series(r);
    default: return -ct_cos_series(r);
  }
}

template <int R>
struct TwTable {
  float c[R];
  float s[R];
};
template <int R>
constexpr TwTable<R> make_tw_table() {
  TwTable<R> t{};
  for (int m = 0; m < R; m++) {
    t.c[m] = (float)ct_cos2pi(m, R);
    t.s[m] = (float)ct_sin2pi(m, R);
  }
  return t;
}
// cos / sin of 2 pi m / R for the composite codelets (m is a constant after unrolling)
template <int R>
struct TwG {
  static __device__ __forceinline__ float c(int m) {
    constexpr TwTable<R> t = make_tw_table<R>();
    return t.c[m];
  }
  static __device__ __forceinline__ float s(int m) {
    constexpr TwTable<R> t = make_tw_table<R>();
    return t.s[m];
  }
};

// Factor split of a composite radix: A = 4 when it divides R (and R > 8), else the
// smallest of 3, 5, 2, 7 that divides.
constexpr int codelet_split(int R) {
  return (R % 4 == 0 && R > 8) ? 4 : (R % 3 == 0) ? 3 : (R % 5 == 0) ? 5 : (R % 2 == 0) ? 2 : 7;
}

template <int R>
struct Dft {
  static __device__ __forceinline__ void run(float2* v, float s) {
    constexpr int A = codelet_split(R);
    dft_composite<A, R / A, R, TwG<R>>(v, s);
  }
};

// ------------------------------------------------------------------ the two passes

// Pass 1 on item t < N2: ld(t, m) reads position t + N2 m, st(t, k2, v) writes position
// t + N2 k2 (the same set of positions).
template <int N1, int N2, int DIR, class Load, class Store>
__device__ __forceinline__ void four_step_pass1(int t, const float2* tw, Load ld, Store st) {
  float2 v[N1];
#pragma unroll
  for (int m = 0; m < N1; m++) v[m] = ld(t, m);
  Dft<N1>::run(v, (float)DIR);
#pragma unroll
  for (int k2 = 1; k2 < N1; k2++) {
    float2 w = tw[t * k2];   // t k2 < N1 N2
    if (DIR > 0) w.y = -w.y;
    v[k2] = cmul(v[k2], w);
  }
#pragma unroll
  for (int k2 = 0; k2 < N1; k2++) st(t, k2, v[k2]);
}

// Pass 2 on item k2 < N1: ld(k2, t) reads position t + N2 k2; v[k1] is output k2 + N1 k1.
template <int N1, int N2, int DIR, class Load>
__device__ __forceinline__ void four_step_pass2(int k2, Load ld, float2 (&v)[N2]) {
#pragma unroll
  for (int t = 0; t < N2; t++) v[t] = ld(k2, t);
  Dft<N2>::run(v, (float)DIR);
}

}  // namespace crava
