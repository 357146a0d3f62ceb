// Shared-memory mixed-radix Stockham FFT on a set of lines held by one CTA.
//
// Replaces the FFTW 2.1.2 codelets the reference calls through rfftw3d
// (libs/fft/fftw/fn_*.c, ftw_*.c, generic.c): lengths are the 2,3,5,7-smooth sizes that
// FFTGrid::findClosestFactorableNumber produces (src/fftgrid.cpp:2630-2658).
//
// A transform of length n = r_0 r_1 ... r_{s-1} runs s autosorting (Stockham) stages.
// Stage t with radix R and Ns = r_0...r_{t-1} maps butterfly j (0 <= j < n/R) as
//   v_r   = x[j + r n/R] * w^(r (j mod Ns) n/(Ns R)),   w = e^{sign 2 pi i / n}
//   y     = DFT_R(v)
//   x'[(j - j mod Ns) R + j mod Ns + r Ns] = y_r
// after which x' is in natural order.  Stages alternate between the lines' buffer and a
// scratch buffer of the same layout in shared memory.  Twiddles come from a table of e^{-2 pi i t / n} evaluated in double precision
// on the host and rounded to float (conjugated for inverse transforms).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace crava {

constexpr int kMaxStages = 16;

struct LinePlan {
  int n;
  int nst;
  int8_t radix[kMaxStages];
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// i*s*a for s = +-1
__device__ __forceinline__ float2 cmul_isign(float2 a, float s) { return make_float2(-s * a.y, s * a.x); }

// cos/sin of 2 pi k / R for the odd radices (values of the constants themselves)
#define C3_S 0.86602540378443864676f
#define C5_C1 0.30901699437494742410f
#define C5_S1 0.95105651629515357212f
#define C5_C2 (-0.80901699437494742410f)
#define C5_S2 0.58778525229247312917f
#define C7_C1 0.62348980185873353053f
#define C7_S1 0.78183148246802980871f
#define C7_C2 (-0.22252093395631440429f)
#define C7_S2 0.97492791218182360702f
#define C7_C3 (-0.90096886790241912624f)
#define C7_S3 0.43388373911755812048f
#define SQRT1_2 0.70710678118654752440f

// In-register DFT of length R, y_m = sum_r v_r e^{sign 2 pi i r m / R}.
template <int R>
struct Dft;

template <>
struct Dft<2> {
  static __device__ __forceinline__ void run(float2* v, float) {
    float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <>
struct Dft<3> {
  static __device__ __forceinline__ void run(float2* v, float s) {
    float2 t1 = cadd(v[1], v[2]);
    float2 t2 = csub(v[1], v[2]);
    float2 m = make_float2(v[0].x - 0.5f * t1.x, v[0].y - 0.5f * t1.y);
    float2 r = cmul_isign(cscale(t2, C3_S), s);
    v[0] = cadd(v[0], t1);
    v[1] = cadd(m, r);
    v[2] = csub(m, r);
  }
};

template <>
struct Dft<4> {
  static __device__ __forceinline__ void run(float2* v, float s) {
    float2 a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
    float2 c = cadd(v[1], v[3]), d = cmul_isign(csub(v[1], v[3]), s);
    v[0] = cadd(a, c);
    v[2] = csub(a, c);
    v[1] = cadd(b, d);
    v[3] = csub(b, d);
  }
};

template <>
struct Dft<5> {
  static __device__ __forceinline__ void run(float2* v, float s) {
    float2 a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
    float2 a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
    float2 x0 = v[0];
    float2 c1 = make_float2(x0.x + C5_C1 * a1.x + C5_C2 * a2.x, x0.y + C5_C1 * a1.y + C5_C2 * a2.y);
    float2 c2 = make_float2(x0.x + C5_C2 * a1.x + C5_C1 * a2.x, x0.y + C5_C2 * a1.y + C5_C1 * a2.y);
    float2 s1 = cmul_isign(make_float2(C5_S1 * b1.x + C5_S2 * b2.x, C5_S1 * b1.y + C5_S2 * b2.y), s);
    float2 s2 = cmul_isign(make_float2(C5_S2 * b1.x - C5_S1 * b2.x, C5_S2 * b1.y - C5_S1 * b2.y), s);
    v[0] = make_float2(x0.x + a1.x + a2.x, x0.y + a1.y + a2.y);
    v[1] = cadd(c1, s1);
    v[4] = csub(c1, s1);
    v[2] = cadd(c2, s2);
    v[3] = csub(c2, s2);
  }
};

template <>
struct Dft<7> {
  static __device__ __forceinline__ void run(float2* v, float s) {
    float2 a1 = cadd(v[1], v[6]), b1 = csub(v[1], v[6]);
    float2 a2 = cadd(v[2], v[5]), b2 = csub(v[2], v[5]);
    float2 a3 = cadd(v[3], v[4]), b3 = csub(v[3], v[4]);
    float2 x0 = v[0];
    // m = 1, 2, 3: cos terms sum a_r cos(2 pi r m/7), sin terms b_r sin(2 pi r m/7)
    float2 c1 = make_float2(x0.x + C7_C1 * a1.x + C7_C2 * a2.x + C7_C3 * a3.x,
                            x0.y + C7_C1 * a1.y + C7_C2 * a2.y + C7_C3 * a3.y);
    float2 c2 = make_float2(x0.x + C7_C2 * a1.x + C7_C3 * a2.x + C7_C1 * a3.x,
                            x0.y + C7_C2 * a1.y + C7_C3 * a2.y + C7_C1 * a3.y);
    float2 c3 = make_float2(x0.x + C7_C3 * a1.x + C7_C1 * a2.x + C7_C2 * a3.x,
                            x0.y + C7_C3 * a1.y + C7_C1 * a2.y + C7_C2 * a3.y);
    // sin(2 pi r m / 7): m=1: S1 S2 S3; m=2: S2 -S3 -S1; m=3: S3 -S1 S2
    float2 s1 = cmul_isign(make_float2(C7_S1 * b1.x + C7_S2 * b2.x + C7_S3 * b3.x,
                                       C7_S1 * b1.y + C7_S2 * b2.y + C7_S3 * b3.y), s);
    float2 s2 = cmul_isign(make_float2(C7_S2 * b1.x - C7_S3 * b2.x - C7_S1 * b3.x,
                                       C7_S2 * b1.y - C7_S3 * b2.y - C7_S1 * b3.y), s);
    float2 s3 = cmul_isign(make_float2(C7_S3 * b1.x - C7_S1 * b2.x + C7_S2 * b3.x,
                                       C7_S3 * b1.y - C7_S1 * b2.y + C7_S2 * b3.y), s);
    v[0] = make_float2(x0.x + a1.x + a2.x + a3.x, x0.y + a1.y + a2.y + a3.y);
    v[1] = cadd(c1, s1);
    v[6] = csub(c1, s1);
    v[2] = cadd(c2, s2);
    v[5] = csub(c2, s2);
    v[3] = cadd(c3, s3);
    v[4] = csub(c3, s3);
  }
};

template <>
struct Dft<8> {
  static __device__ __forceinline__ void run(float2* v, float s) {
    // radix-2 split: DFT4 of even and odd, odd twiddled by e^{sign 2 pi i m/8}
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    Dft<4>::run(e, s);
    Dft<4>::run(o, s);
    // w1 = (1 + s i)/sqrt2, w2 = s i, w3 = (-1 + s i)/sqrt2
    float2 o1 = make_float2(SQRT1_2 * (o[1].x - s * o[1].y), SQRT1_2 * (o[1].y + s * o[1].x));
    float2 o2 = cmul_isign(o[2], s);
    float2 o3 = make_float2(SQRT1_2 * (-o[3].x - s * o[3].y), SQRT1_2 * (-o[3].y + s * o[3].x));
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], o1);
    v[5] = csub(e[1], o1);
    v[2] = cadd(e[2], o2);
    v[6] = csub(e[2], o2);
    v[3] = cadd(e[3], o3);
    v[7] = csub(e[3], o3);
  }
};

// Composite radix R = A*B in registers (Cooley-Tukey): B-point DFTs over the A
// decimated subsequences v[r1 + A r2], twiddles e^{sign 2 pi i r1 k2 / R}, A-point DFTs,
// output X[k2 + B k1].  TW::c(m), TW::s(m): cos and sin of 2 pi m / R.
template <int A, int B, int R, class TW>
__device__ __forceinline__ void dft_composite(float2* v, float s) {
  float2 u[A][B];
#pragma unroll
  for (int r1 = 0; r1 < A; r1++) {
#pragma unroll
    for (int r2 = 0; r2 < B; r2++) u[r1][r2] = v[r1 + A * r2];
    Dft<B>::run(u[r1], s);
#pragma unroll
    for (int k2 = 1; k2 < B; k2++) {
      const int m = (r1 * k2) % R;
      if (r1 > 0) u[r1][k2] = cmul(u[r1][k2], make_float2(TW::c(m), s * TW::s(m)));
    }
  }
#pragma unroll
  for (int k2 = 0; k2 < B; k2++) {
    float2 t[A];
#pragma unroll
    for (int r1 = 0; r1 < A; r1++) t[r1] = u[r1][k2];
    Dft<A>::run(t, s);
#pragma unroll
    for (int k1 = 0; k1 < A; k1++) v[k2 + B * k1] = t[k1];
  }
}

struct Tw6 {
  static __device__ __forceinline__ float c(int m) {
    constexpr float t[6] = {1.f, 0.5f, -0.5f, -1.f, -0.5f, 0.5f};
    return t[m];
  }
  static __device__ __forceinline__ float s(int m) {
    constexpr float t[6] = {0.f, 0.86602540378443865f, 0.86602540378443865f, 0.f, -0.86602540378443865f,
                            -0.86602540378443865f};
    return t[m];
  }
};
struct Tw9 {
  static __device__ __forceinline__ float c(int m) {
    constexpr float t[9] = {1.f, 0.76604444311897804f, 0.17364817766693035f, -0.5f, -0.93969262078590838f,
                            -0.93969262078590838f, -0.5f, 0.17364817766693035f, 0.76604444311897804f};
    return t[m];
  }
  static __device__ __forceinline__ float s(int m) {
    constexpr float t[9] = {0.f, 0.64278760968653933f, 0.98480775301220806f, 0.86602540378443865f,
                            0.34202014332566873f, -0.34202014332566873f, -0.86602540378443865f,
                            -0.98480775301220806f, -0.64278760968653933f};
    return t[m];
  }
};
struct Tw16 {
  static __device__ __forceinline__ float c(int m) {
    constexpr float t[16] = {1.f, 0.92387953251128676f, 0.70710678118654752f, 0.38268343236508977f, 0.f,
                             -0.38268343236508977f, -0.70710678118654752f, -0.92387953251128676f, -1.f,
                             -0.92387953251128676f, -0.70710678118654752f, -0.38268343236508977f, 0.f,
                             0.38268343236508977f, 0.70710678118654752f, 0.92387953251128676f};
    return t[m];
  }
  static __device__ __forceinline__ float s(int m) {
    constexpr float t[16] = {0.f, 0.38268343236508977f, 0.70710678118654752f, 0.92387953251128676f, 1.f,
                             0.92387953251128676f, 0.70710678118654752f, 0.38268343236508977f, 0.f,
                             -0.38268343236508977f, -0.70710678118654752f, -0.92387953251128676f, -1.f,
                             -0.92387953251128676f, -0.70710678118654752f, -0.38268343236508977f};
    return t[m];
  }
};

template <>
struct Dft<6> {
  static __device__ __forceinline__ void run(float2* v, float s) { dft_composite<2, 3, 6, Tw6>(v, s); }
};
template <>
struct Dft<9> {
  static __device__ __forceinline__ void run(float2* v, float s) { dft_composite<3, 3, 9, Tw9>(v, s); }
};
template <>
struct Dft<16> {
  static __device__ __forceinline__ void run(float2* v, float s) { dft_composite<4, 4, 16, Tw16>(v, s); }
};

// q = x / d, r = x % d for 0 <= x < 2^22 and d >= 1, with rcp = 1/d rounded to float:
// the float quotient is within one of the exact one and a single correction fixes it.
__device__ __forceinline__ int fdivmod(int x, int d, float rcp, int& r) {
  int q = __float2int_rz(__int2float_rn(x) * rcp);
  r = x - q * d;
  if (r < 0) { q -= 1; r += d; }
  else if (r >= d) { q += 1; r -= d; }
  return q;
}

// 32-bit shared-memory addressing: stages address their buffers by shared-window byte
// addresses so that index arithmetic stays 32-bit.
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ float2 lds2(uint32_t a) {
  float2 v;
  asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(a));
  return v;
}
__device__ __forceinline__ void sts2(uint32_t a, float2 v) {
  asm volatile("st.shared.v2.f32 [%0], {%1, %2};" ::"r"(a), "f"(v.x), "f"(v.y) : "memory");
}

// Thread-to-line mapping shared by every stage of one fft_lines call in LC mode:
// thread t starts at line t % nlines, butterfly row t / nlines, and advances by T.
// cp.async (global -> shared without registers), 8 bytes; the zero-filling form with
// valid = false writes 8 zero bytes and reads nothing.
__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src) : "memory");
}
// zero-filling form: src_bytes 0 writes 8 zero bytes and reads nothing
__device__ __forceinline__ void cp_async8_zfill(uint32_t dst, const void* src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src), "r"(valid ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

// L2 prefetch of the global bytes [p, p + n) of a buffer [b0, b1) that holds them: the range
// is widened to 16-byte boundaries (the bulk prefetch's alignment rule) inside the buffer and
// the bytes that cannot be so widened are left out; a hint with no effect on the values.
__device__ __forceinline__ void l2_prefetch(const void* p, size_t n, const void* b0, const void* b1) {
  uintptr_t a = reinterpret_cast<uintptr_t>(p) & ~(uintptr_t)15;
  uintptr_t e = (reinterpret_cast<uintptr_t>(p) + n + 15) & ~(uintptr_t)15;
  if (a < reinterpret_cast<uintptr_t>(b0)) a += 16;
  if (e > reinterpret_cast<uintptr_t>(b1)) e -= 16;
  if (e > a) {
    const size_t ga = __cvta_generic_to_global(reinterpret_cast<const void*>(a));
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(ga), "r"((uint32_t)(e - a)) : "memory");
  }
}
// L2 prefetch of the cache line holding global address p (an ordinary load-unit request, no
// bulk-copy unit); p must lie inside an allocation.
__device__ __forceinline__ void l2_prefetch_line(const void* p) {
  asm volatile("prefetch.global.L2 [%0];\n" ::"l"(__cvta_generic_to_global(p)));
}
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

struct LcMap {
  int f0, s0, df, ds;
};

// One Stockham stage over nlines lines from `in` to `out` (shared-window byte addresses).
// Element p of line l sits at in + 8 (l*ls + p*psi) and out + 8 (l*ls + p*pso).  LC
// (lines contiguous): consecutive threads take consecutive lines of one butterfly index
// j; otherwise consecutive j of one line.  The (line, j, j mod Ns, j / Ns) of a thread's
// butterflies advance incrementally after a few reciprocal-based divisions per stage.
// DIR = -1 forward, +1 inverse.
template <int R, bool LC, int DIR>
__device__ __forceinline__ void fft_stage(uint32_t in, uint32_t out, int nlines, int ls, int psi, int pso, int n,
                                          int Ns, const LcMap& mp, uint32_t tw) {
  constexpr float sign = (float)DIR;
  const int nb = n / R;
  const int total = nlines * nb;
  const int T = blockDim.x;
  const float rNs = __frcp_rn((float)Ns);
  int tmp;
  const int nbh = fdivmod(nb, Ns, rNs, tmp);  // nb / Ns (exact) = n / (Ns R), the twiddle stride
  const uint32_t istep = 8u * (uint32_t)(nb * psi);   // bytes between the R inputs
  const uint32_t ostep = 8u * (uint32_t)(Ns * pso);   // bytes between the R outputs
  const uint32_t tstep = 8u * (uint32_t)nbh;          // twiddle bytes per unit of r*k
  int idx = threadIdx.x;
  int line, j, df, ds;
  if (LC) {
    line = mp.f0; j = mp.s0; df = mp.df; ds = mp.ds;
  } else {
    const float rnb = __frcp_rn((float)nb);
    int f;
    line = fdivmod(idx, nb, rnb, f);
    j = f;
    ds = fdivmod(T, nb, rnb, df);
  }
  int k;
  int jh = fdivmod(j, Ns, rNs, k);
  const int dj = LC ? ds : df;
  int dk;
  const int djh = fdivmod(dj, Ns, rNs, dk);
  const int RNs = R * Ns;
  for (; idx < total; idx += T) {
    uint32_t a = in + 8u * (uint32_t)(line * ls + j * psi);
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = lds2(a + r * istep);
    if (Ns > 1) {
      const uint32_t kt = (uint32_t)k * tstep;  // byte offset of e^{-2 pi i k/(Ns R)}
#pragma unroll
      for (int r = 1; r < R; r++) {
        float2 w = lds2(tw + r * kt);
        if (DIR > 0) w.y = -w.y;  // table holds e^{-2 pi i t/n}
        v[r] = cmul(v[r], w);
      }
    }
    Dft<R>::run(v, sign);
    uint32_t o = out + 8u * (uint32_t)(line * ls + (jh * RNs + k) * pso);
#pragma unroll
    for (int r = 0; r < R; r++) sts2(o + r * ostep, v[r]);
    if (LC) {
      line += df;
      int carry = line >= nlines;
      if (carry) line -= nlines;
      j += dj + carry;
      k += dk + carry;
      jh += djh;
      if (k >= Ns) { k -= Ns; jh += 1; }
    } else {
      j += dj;
      k += dk;
      jh += djh;
      if (k >= Ns) { k -= Ns; jh += 1; }
      line += ds;
      if (j >= nb) { j -= nb; jh -= nbh; line += 1; }
    }
  }
  __syncthreads();
}

// Full transform of nlines lines of length pl.n.  The lines start in `buf` (point stride
// ps) and end there; `scratch` (dense, point stride nlines when LC, line stride n
// otherwise) holds the odd stages.  DIR = -1 forward, +1 inverse, unnormalised both ways
// like FFTW.  tw: the length-n table of e^{-2 pi i t/n} in shared memory.  The caller
// synchronises before the call; the function returns after a barrier.  Stages run
// grouped by radix in the fixed order 16.., 8.., 4, 2, 9.., 3.., 6.., 5.., 7.. (any order
// of the radices gives the same transform).  R16 = false compiles without the radix-16
// stage (for kernels capped at 64 registers; their plans never contain it).
template <bool LC, int DIR, bool R16 = true>
__device__ __forceinline__ void fft_lines(float2* buf, float2* scratch, int nlines, int ls, int ps,
                                          const LinePlan& pl, const float2* tw) {
  int Ns = 1;
  const int n = pl.n;
  int c16 = 0, c8 = 0, c4 = 0, c2 = 0, c9 = 0, c3 = 0, c6 = 0, c5 = 0, c7 = 0;
  for (int s = 0; s < pl.nst; s++) {
    int R = pl.radix[s];
    c16 += R == 16; c8 += R == 8; c4 += R == 4; c2 += R == 2; c9 += R == 9; c3 += R == 3;
    c6 += R == 6; c5 += R == 5; c7 += R == 7;
  }
  LcMap mp{0, 0, 0, 0};
  if (LC) {
    const float rl = __frcp_rn((float)nlines);
    mp.s0 = fdivmod(threadIdx.x, nlines, rl, mp.f0);
    mp.ds = fdivmod(blockDim.x, nlines, rl, mp.df);
  }
  const uint32_t b = smem_addr(buf), sc = smem_addr(scratch), t = smem_addr(tw);
  // scratch layout: LC -> element (l, p) at l + p*nlines; else at l*n + p
  const int sps = LC ? nlines : 1;
  const int lsx = LC ? 1 : ls;
  bool in_buf = true;
#define CRAVA_STAGE(RR)                                                                       \
  {                                                                                           \
    if (in_buf) fft_stage<RR, LC, DIR>(b, sc, nlines, lsx, ps, sps, n, Ns, mp, t);            \
    else fft_stage<RR, LC, DIR>(sc, b, nlines, lsx, sps, ps, n, Ns, mp, t);                   \
    Ns *= RR;                                                                                 \
    in_buf = !in_buf;                                                                         \
  }
  if (R16) {  // plans built without radix 16 leave c16 == 0
#pragma unroll 1
    for (int q = 0; q < c16; q++) CRAVA_STAGE(16)
  }
#pragma unroll 1
  for (int q = 0; q < c8; q++) CRAVA_STAGE(8)
  if (c4) CRAVA_STAGE(4)
  if (c2) CRAVA_STAGE(2)
#pragma unroll 1
  for (int q = 0; q < c9; q++) CRAVA_STAGE(9)
#pragma unroll 1
  for (int q = 0; q < c3; q++) CRAVA_STAGE(3)
#pragma unroll 1
  for (int q = 0; q < c6; q++) CRAVA_STAGE(6)
#pragma unroll 1
  for (int q = 0; q < c5; q++) CRAVA_STAGE(5)
#pragma unroll 1
  for (int q = 0; q < c7; q++) CRAVA_STAGE(7)
#undef CRAVA_STAGE
  if (!in_buf) {  // odd number of stages: copy back
    if (LC) {
      const float rl = __frcp_rn((float)nlines);
      for (int e = threadIdx.x; e < nlines * n; e += blockDim.x) {
        int l;
        int p = fdivmod(e, nlines, rl, l);
        sts2(b + 8u * (uint32_t)(l + p * ps), lds2(sc + 8u * (uint32_t)e));
      }
    } else {
      const float rn = __frcp_rn((float)n);
      for (int e = threadIdx.x; e < nlines * n; e += blockDim.x) {
        int p;
        int l = fdivmod(e, n, rn, p);
        sts2(b + 8u * (uint32_t)(l * ls + p * ps), lds2(sc + 8u * (uint32_t)e));
      }
    }
    __syncthreads();
  }
}

}  // namespace crava
