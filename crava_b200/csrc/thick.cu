// Non-constant-thickness pre-processing of the seismic data (sm_100a):
//
//   AVOInversion::divideDataByScaleWavelet + computeAdjustmentFactor
//     (src/avoinversion.cpp:484-719): every trace (i, j) of the padded grid is tapered in
//     the z padding, transformed along z, multiplied inside the band by a per-trace factor
//     that swaps the trace's stretched wavelet for a global one, and transformed back;
//   FFTGrid::interpolateSeismic / interpolateTrace / extrapolateSeismic
//     (src/fftgrid.cpp:2349-2516): traces whose energy is at or below the threshold are
//     replaced by the mean of their good neighbours, and every trace outside the box of
//     good traces (the lateral padding included) by a tapered copy of its mirror trace.
//
// The trace transform packs two real traces (x = 2m, 2m + 1, adjacent floats) into one
// complex line, transforms W such lines of one (j, angle) together in shared memory with
// the Stockham engine, separates the two half spectra, multiplies each by its own factor,
// recombines them and transforms back: one read and one write of the grid.  The factor is
// evaluated per (trace, kz) in the reference's float arithmetic with explicitly rounded
// operations (no contraction into FMA), so it equals the reference's float value for the
// same tables.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <vector>

#include "kernels.cuh"

namespace crava {

namespace {

__device__ __forceinline__ float sq2(float2 v) { return __fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y)); }

// x / float(sqrt(float(nzp))) correctly rounded; a multiplication when the divisor is a
// power of two (nzp = 4^m), which rounds the same exact quotient once
__device__ __forceinline__ float div_rsq(const ThickParams& P, float x) {
  return P.inv_rsq != 0.f ? __fmul_rn(x, P.inv_rsq) : __fdiv_rn(x, P.rsq);
}

// Wavelet::getCAmp(k, scale) for k < cnzp (src/wavelet.cpp:337-382): the spectrum of the
// wavelet stretched by `scale`, linear interpolation at k / scale, divided by scale; the
// spectrum's value at bin m is at(m).
template <class At>
__device__ __forceinline__ float2 interp_scaled(int cnzp, int k, float scale, At at) {
  const float om = __fdiv_rn((float)k, scale);
  if (!(om < (float)cnzp)) return make_float2(0.f, 0.f);
  const int lo = (int)floorf(om);
  int hi = lo + 1;
  if (hi >= cnzp) hi -= 1;
  const float d = __fsub_rn(om, (float)lo);
  const float e = __fsub_rn(1.f, d);
  const float2 a = at(lo), b = at(hi);
  const float re = __fadd_rn(__fmul_rn(a.x, e), __fmul_rn(b.x, d));
  const float im = __fadd_rn(__fmul_rn(a.y, e), __fmul_rn(b.y, d));
  return make_float2(__fdiv_rn(re, scale), __fdiv_rn(im, scale));
}

// interp_scaled's last step for two spectra at the same position: (a e + b d) / scale.
__device__ __forceinline__ float2 lerp_scaled(float2 a, float2 b, float e, float d, float scale) {
  const float re = __fadd_rn(__fmul_rn(a.x, e), __fmul_rn(b.x, d));
  const float im = __fadd_rn(__fmul_rn(a.y, e), __fmul_rn(b.y, d));
  return make_float2(__fdiv_rn(re, scale), __fdiv_rn(im, scale));
}

__device__ __forceinline__ float2 camp_scaled(const float2* c, int cnzp, int k, float scale) {
  return interp_scaled(cnzp, k, scale, [&](int m) { return __ldg(c + m); });
}

// Wavelet1D::shiftAndScale (src/wavelet1D.cpp:580-602) at bin m: the multiplier
// float(gain cos(2 pi iShift m / nzp)) + i float(gain sin(-2 pi iShift m / nzp)), with the
// angle and the products in double as the reference forms them, applied to c in float.
__device__ __forceinline__ float2 shift_scale(float2 c, float ish, float gain, int m, int nzp) {
  const double a = 2.0 * (3.14159265358979323846 * (double)ish * (double)m) / (double)(float)nzp;
  double sn, cs;
  sincos(a, &sn, &cs);
  const float mr = (float)((double)gain * cs), mi = (float)((double)gain * -sn);
  return make_float2(__fsub_rn(__fmul_rn(mr, c.x), __fmul_rn(mi, c.y)),
                     __fadd_rn(__fmul_rn(mi, c.x), __fmul_rn(mr, c.y)));
}

// computeAdjustmentFactor (src/avoinversion.cpp:630-719) at one kz < cnzp for a trace
// whose wavelet is stretched by sf; local wavelet = global wavelet (1D wavelet without
// local shift or gain grids), so eSkGlob uses the unstretched spectrum of the same tables.
// The quantities of the global wavelet (wGlob2Adj, tolFac*wGlob2Adj and the quotient
// wGlob2Adj / (tau2 wGlob2 + sigma2Glob)) do not depend on the trace: the host evaluates
// them per (angle, kz) with the same float operations (glob[] = {tg, q}).
__device__ __forceinline__ float2 adjustment(const ThickParams& P, int l, int k, float sf) {
  const int cn = P.cnzp;
  const float2* wa = P.wamp + (size_t)l * cn;
  const float2* es = P.es3 + (size_t)l * cn;
  const float wn2 = P.wn2[l], wnc = P.wnc, ev = P.err_var[l];
  const float2 wLoc = camp_scaled(wa, cn, k, sf);
  const float wLoc2 = sq2(wLoc);
  const float sL = __fadd_rn(__fdiv_rn(wLoc2, wn2), sq2(camp_scaled(es, cn, k, sf)));
  const float c = __fmul_rn(__fsub_rn(1.f, wnc), 0.5f);
  float s2L = __fmul_rn(ev, __fadd_rn(wnc, __fmul_rn(c, sL)));
  const float tau2 = __ldg(P.tau2 + (size_t)l * cn + k);
  const float2 glob = __ldg(P.glob + (size_t)l * cn + k);
  const float tm = __fmul_rn(0.05f, P.modW[l]);
  float wL2A = wLoc2;
  if (wLoc2 < tm) wL2A = __fmul_rn(0.5f, __fadd_rn(wLoc2, tm));
  if (wL2A < glob.x) {
    wL2A = __fmul_rn(0.5f, __fadd_rn(wLoc2, glob.x));
    s2L = __fmul_rn(s2L, __fdiv_rn(wL2A, wLoc2));
  }
  const float dL = __fadd_rn(__fmul_rn(tau2, wL2A), s2L);
  return make_float2(__fdiv_rn(__fdiv_rn(wLoc.x, dL), glob.y), __fdiv_rn(__fdiv_rn(wLoc.y, dL), glob.y));
}

// The local wavelet of one trace: shift ish (samples) and gain gn of shiftAndScale, and for
// 3D wavelets the dip adjustment (multiplyer, Halpha), the norm^2 of the adjusted wavelet and
// gamma, which band-normalises its errorSmooth3 given the normalised table.  1D wavelets:
// mult 1, Halpha 0, the global norm^2 and gamma 1, under which every factor below is an
// exact 1.
struct LocalWavelet {
  float ish, gn;
  double mult;
  float H, wn2, gam;
};

// Wavelet1D::adjustForAmplitudeEffect (src/wavelet1D.cpp:605-636) at bin m: the factor
// float(multiplyer * float(exp(-pi omega Halpha))) with omega = m / double(nzp dz 1e-3), or
// float(multiplyer) when Halpha <= 0.
__device__ __forceinline__ float dip_factor(double den, int m, double mult, float H) {
  if (!(H > 0.f)) return (float)mult;
  const double om = __ddiv_rn((double)m, den);
  const float am = (float)exp(__dmul_rn(__dmul_rn(-3.14159265358979323846, om), (double)H));
  return (float)__dmul_rn(mult, (double)am);
}

// The local wavelet's spectrum at bin m: the global one through the dip adjustment
// (extractLocalWaveletByDip1D, src/wavelet3D.cpp:436-459) and shiftAndScale
// (createLocalWavelet1D, src/wavelet1D.cpp:518-526, src/wavelet3D.cpp:347-373).  Its
// errorSmooth3 is the normalised table's entry times the same dip factor and gamma, turned by
// the shift's unit-modulus multiplier (the band normalisation takes the gain out; the
// RMISSING entry at cnzp - 1 stays).  The reference re-transforms the local wavelet between
// these steps (the amplitude adjustment and the difference constructors work on its
// samples); here the spectra are used directly.
__device__ __forceinline__ float2 local_wavelet(const ThickParams& P, int l, int m, const LocalWavelet& w) {
  float2 c = __ldg(P.wamp + (size_t)l * P.cnzp + m);
  if (P.w3_mult) {
    const float f = dip_factor(P.w3_den, m, w.mult, w.H);
    c = make_float2(__fmul_rn(c.x, f), __fmul_rn(c.y, f));
  }
  return shift_scale(c, w.ish, w.gn, m, P.nzp);
}

// The local wavelet's spectrum (w) and errorSmooth3 (e) at bin m, as local_wavelet and its
// errorSmooth3 above, sharing the dip factor and the shift's angle (one double exp and one
// double sincos per bin; the same float operations as evaluating them apart).
struct LocalBin {
  float2 w, e;
};

__device__ __forceinline__ LocalBin local_pair(const ThickParams& P, int l, int m, const LocalWavelet& w) {
  const int cn = P.cnzp;
  float2 c = __ldg(P.wamp + (size_t)l * cn + m);
  float2 s = m < cn - 1 ? __ldg(P.es3 + (size_t)l * cn + m) : P.es3_last[l];
  if (P.w3_mult) {
    const float f = dip_factor(P.w3_den, m, w.mult, w.H);
    c = make_float2(__fmul_rn(c.x, f), __fmul_rn(c.y, f));
    s = make_float2(__fmul_rn(__fmul_rn(s.x, f), w.gam), __fmul_rn(__fmul_rn(s.y, f), w.gam));
  }
  const double a = 2.0 * (3.14159265358979323846 * (double)w.ish * (double)m) / (double)(float)P.nzp;
  double sn, cs;
  sincos(a, &sn, &cs);
  const float mr = (float)((double)w.gn * cs), mi = (float)((double)w.gn * -sn);   // gain gn
  const float nr = (float)cs, ni = (float)-sn;                                      // gain 1
  LocalBin r;
  r.w = make_float2(__fsub_rn(__fmul_rn(mr, c.x), __fmul_rn(mi, c.y)), __fadd_rn(__fmul_rn(mi, c.x), __fmul_rn(mr, c.y)));
  r.e = make_float2(__fsub_rn(__fmul_rn(nr, s.x), __fmul_rn(ni, s.y)), __fadd_rn(__fmul_rn(ni, s.x), __fmul_rn(nr, s.y)));
  if (m == cn - 1) {
    r.e.y = -99999.0f;
    if (!(P.nzp & 1)) r.e.x = -99999.0f;
  }
  return r;
}

// computeAdjustmentFactor (src/avoinversion.cpp:630-719) with a trace's local wavelet: wLoc
// and eSkLoc from the local spectra stretched by sf, eSkGlob from the local spectra
// unstretched (wLocal->getCAmp(k)), wGlob from the global wavelet (the 1D wavelet itself, or
// for 3D wavelets Wavelet3D::getGlobalWavelet, whose norm the host puts into modW); the
// global wavelet's quotient then depends on the trace and is formed here with the host's
// float operations.
__device__ __forceinline__ float2 adjustment_local(const ThickParams& P, int l, int k, float sf, const LocalWavelet& w) {
  const int cn = P.cnzp;
  const float wn2 = w.wn2, wnc = P.wnc, ev = P.err_var[l];
  // getCAmp(k, sf) of both local spectra (interp_scaled's steps, one position)
  float2 wLoc = make_float2(0.f, 0.f), eLoc = wLoc;
  const float om = __fdiv_rn((float)k, sf);
  if (om < (float)cn) {
    const int lo = (int)floorf(om);
    int hi = lo + 1;
    if (hi >= cn) hi -= 1;
    const float d = __fsub_rn(om, (float)lo);
    const float e = __fsub_rn(1.f, d);
    const LocalBin A = local_pair(P, l, lo, w), B = local_pair(P, l, hi, w);
    wLoc = lerp_scaled(A.w, B.w, e, d, sf);
    eLoc = lerp_scaled(A.e, B.e, e, d, sf);
  }
  const LocalBin K = local_pair(P, l, k, w);
  const float wLoc2 = sq2(wLoc);
  const float sL = __fadd_rn(__fdiv_rn(wLoc2, wn2), sq2(eLoc));
  const float c = __fmul_rn(__fsub_rn(1.f, wnc), 0.5f);
  float s2L = __fmul_rn(ev, __fadd_rn(wnc, __fmul_rn(c, sL)));
  const float sG = __fadd_rn(__fdiv_rn(sq2(K.w), wn2), sq2(K.e));
  const float s2G = __fmul_rn(ev, __fadd_rn(wnc, __fmul_rn(c, sG)));
  const float wGlob2 = sq2(__ldg((P.wglob ? P.wglob : P.wamp) + (size_t)l * cn + k));
  const float tau2 = __ldg(P.tau2 + (size_t)l * cn + k);
  const float tm = __fmul_rn(0.05f, P.modW[l]);
  const float wG2A = wGlob2 < tm ? __fmul_rn(0.5f, __fadd_rn(wGlob2, tm)) : wGlob2;
  const float tg = __fmul_rn(0.05f, wG2A);
  const float q = __fdiv_rn(wG2A, __fadd_rn(__fmul_rn(tau2, wGlob2), s2G));
  float wL2A = wLoc2;
  if (wLoc2 < tm) wL2A = __fmul_rn(0.5f, __fadd_rn(wLoc2, tm));
  if (wL2A < tg) {
    wL2A = __fmul_rn(0.5f, __fadd_rn(wLoc2, tg));
    s2L = __fmul_rn(s2L, __fdiv_rn(wL2A, wLoc2));
  }
  const float dL = __fadd_rn(__fmul_rn(tau2, wL2A), s2L);
  return make_float2(__fdiv_rn(__fdiv_rn(wLoc.x, dL), q), __fdiv_rn(__fdiv_rn(wLoc.y, dL), q));
}

// The index of the unpadded trace whose local wavelet a padded trace uses
// (src/avoinversion.cpp:525-543).
__device__ __forceinline__ int wavelet_index(int i, int n, int np) {
  if (i > 3 * n - 1) i = 0;
  if (i > (np + n) / 2) i = np - i;
  if (i >= n) i = 2 * n - i - 1;
  return i;
}

// One CTA: W complex lines (2W traces x = 2(m0 + w) + {0, 1}) of row j of angle blockIdx.z.
// Mode 0 divides every padded trace by its scale wavelet; mode 1 convolves the traces
// i < nx, j < ny with their local wavelets (multiplyDataByScaleWaveletAndWriteToFile,
// src/avoinversion.cpp:743-776: 1/sqrt(nzp), r2c, times the conjugate of
// getCAmp(k, relThick) at every kz, c2r, 1/sqrt(nzp)) and leaves the other traces as they are.
// LOCAL: mode 0 with local wavelets (shift/gain grids or 3D wavelets), whose per-trace factor
// needs more registers than the tabulated one; a separate instantiation keeps the plain
// division at its own register count.
template <bool LOCAL>
__global__ void __launch_bounds__(256) k_thick_divide(const __grid_constant__ ThickParams P) {
  extern __shared__ float2 sm[];
  const int nzp = P.nzp, W = P.W, lw = P.logW, half = nzp / 2;
  float2* tw = sm;
  float2* R = tw + nzp;
  float2* SC = R + (size_t)W * nzp;
  __shared__ float s_sf[2 * 32];
  __shared__ double s_df[2 * 32];
  __shared__ LocalWavelet s_lw[2 * 32];            // the traces' local wavelets
  __shared__ int s_live[2 * 32];   // the trace has a nonzero tapered sample
  const int tid = threadIdx.x, T = blockDim.x;
  const int j = blockIdx.y, l = blockIdx.z;
  const int m0 = blockIdx.x * W;
  const bool conv = P.mode == 1;
  const int nlive = conv ? P.nx : P.nxp;   // traces this mode reads and writes
  float* g = P.grid[l];
  const size_t kstride = (size_t)P.nyp * P.rnxp;
  float* row = g + (size_t)j * P.rnxp;
  for (int t = tid; t < nzp; t += T) tw[t] = P.twz[t];
  // per trace: the local wavelet, the stretch sf as getCAmp receives it (divide mode
  // float(relThick * double(localStretch)), src/avoinversion.cpp:557; convolution mode
  // float(relThick) * localStretch, :748; the local stretch is 1 for 1D wavelets) and
  // deltaF = nz*1000 / (relThick * lz * nzp) (:559-560)
  if (tid < 2 * W) {
    const int i = 2 * m0 + tid;
    double rt = 1.0;
    if (P.rel_thick && i < P.nxp) rt = P.rel_thick[(size_t)j * P.nxp + i];
    LocalWavelet lw{0.f, 1.f, 1.0, 0.f, P.wn2[l], 1.f};
    float stretch = 1.f;
    if ((P.wshift || P.w3_mult) && i < P.nxp) {
      const size_t t = (size_t)l * P.nx * P.ny + (size_t)wavelet_index(j, P.ny, P.nyp) * P.nx +
                       wavelet_index(i, P.nx, P.nxp);
      if (P.wshift) {
        lw.ish = P.wshift[t];
        lw.gn = P.wgain[t];
      }
      if (P.w3_mult) {
        const float4 q = P.w3_par[t];
        lw.mult = P.w3_mult[t];
        lw.H = q.x;
        stretch = q.y;
        lw.wn2 = q.z;
        lw.gam = q.w;
      }
    }
    s_lw[tid] = lw;
    s_sf[tid] = conv ? __fmul_rn((float)rt, stretch) : (float)__dmul_rn(rt, (double)stretch);
    s_df[tid] = __ddiv_rn(__dmul_rn((double)P.nz, 1000.0), __dmul_rn(__dmul_rn(rt, P.lz), (double)nzp));
    s_live[tid] = 0;
  }
  __syncthreads();
  // load, 1/sqrt(nzp) and the z taper (:539-551); traces at or beyond nxp load as zero.
  // A trace whose tapered samples are all zero (a dead trace) is stored back as exact
  // zeros, as the reference's own real transform returns it, although the trace sharing
  // its complex line leaks rounding into it.
  // every copy is issued before the first is waited for (cp.async); a line whose second
  // trace lies at nxp (odd nxp) is read by a plain load of its first float
  {
    const uint32_t rb = smem_addr(R);
    for (int e = tid; e < W * nzp; e += T) {
      const int w = e & (W - 1), k = e >> lw;
      const int m = m0 + w;
      const float* p = row + (size_t)k * kstride + 2 * m;
      if (2 * m + 1 < nlive) {
        cp_async8(rb + 8u * (uint32_t)e, p);
      } else {
        R[e] = make_float2(2 * m < nlive ? *p : 0.f, 0.f);
      }
    }
    cp_async_commit();
    cp_async_wait_0();
  }
  __syncthreads();
  for (int e = tid; e < W * nzp; e += T) {
    const int w = e & (W - 1), k = e >> lw;
    float2 v = R[e];
    const float tz = conv ? 1.f : __ldg(P.ztaper + k);
    v.x = __fmul_rn(div_rsq(P, v.x), tz);
    v.y = __fmul_rn(div_rsq(P, v.y), tz);
    if (v.x != 0.f) s_live[2 * w] = 1;
    if (v.y != 0.f) s_live[2 * w + 1] = 1;
    R[e] = v;
  }
  __syncthreads();
  fft_lines<true, -1>(R, SC, W, 1, W, P.zp, tw);
  __syncthreads();
  // half spectra of the two traces, Z = A + iB: A(k) = (Z(k) + conj Z(-k)) / 2,
  // B(k) = (Z(k) - conj Z(-k)) / 2i; factor and band per trace; the c2r of the reference
  // ignores the imaginary parts at DC and Nyquist; Z'(k) = A' + iB', Z'(-k) = conj A' + i conj B'
  for (int e = tid; e < W * (half + 1); e += T) {
    const int w = e & (W - 1), k = e >> lw;
    const int kk = (k == 0) ? 0 : nzp - k;
    const float2 z = R[k * W + w], zc = R[kk * W + w];
    float2 a = make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y - zc.y));
    float2 b = make_float2(0.5f * (z.y + zc.y), -0.5f * (z.x - zc.x));
    const int m = m0 + w;
    float2 fa = make_float2(0.f, 0.f), fb = fa;
    if (conv) {
      // the conjugate of the local wavelet's stretched spectrum (getCAmp returns the
      // conjugate's value, src/avoinversion.cpp:761-768)
      if (2 * m < nlive) {
        const LocalWavelet& lw = s_lw[2 * w];
        const float2 v = interp_scaled(P.cnzp, k, s_sf[2 * w], [&](int q) { return local_wavelet(P, l, q, lw); });
        fa = make_float2(v.x, -v.y);
      }
      if (2 * m + 1 < nlive) {
        const LocalWavelet& lw = s_lw[2 * w + 1];
        const float2 v = interp_scaled(P.cnzp, k, s_sf[2 * w + 1], [&](int q) { return local_wavelet(P, l, q, lw); });
        fb = make_float2(v.x, -v.y);
      }
    } else {
      if (2 * m < P.nxp) {
        const double fk = __dmul_rn(s_df[2 * w], (double)k);
        if (fk < (double)P.high_cut && fk > (double)P.low_cut)
          fa = LOCAL ? adjustment_local(P, l, k, s_sf[2 * w], s_lw[2 * w]) : adjustment(P, l, k, s_sf[2 * w]);
      }
      if (2 * m + 1 < P.nxp) {
        const double fk = __dmul_rn(s_df[2 * w + 1], (double)k);
        if (fk < (double)P.high_cut && fk > (double)P.low_cut)
          fb = LOCAL ? adjustment_local(P, l, k, s_sf[2 * w + 1], s_lw[2 * w + 1])
                     : adjustment(P, l, k, s_sf[2 * w + 1]);
      }
    }
    a = cmul(a, fa);
    b = cmul(b, fb);
    if (k == 0 || 2 * k == nzp) {
      a.y = 0.f;
      b.y = 0.f;
    }
    R[k * W + w] = make_float2(a.x - b.y, a.y + b.x);
    if (kk != k) R[kk * W + w] = make_float2(a.x + b.y, b.x - a.y);
  }
  __syncthreads();
  fft_lines<true, 1>(R, SC, W, 1, W, P.zp, tw);
  __syncthreads();
  for (int e = tid; e < W * nzp; e += T) {
    const int w = e & (W - 1), k = e >> lw;
    const int m = m0 + w;
    if (2 * m >= nlive) continue;
    float* p = row + (size_t)k * kstride + 2 * m;
    const float2 v = R[e];
    float2 o;
    if (conv) o = make_float2(s_live[2 * w] ? __fdiv_rn(v.x, P.rsq_out) : 0.f, s_live[2 * w + 1] ? __fdiv_rn(v.y, P.rsq_out) : 0.f);
    else o = make_float2(s_live[2 * w] ? div_rsq(P, v.x) : 0.f, s_live[2 * w + 1] ? div_rsq(P, v.y) : 0.f);
    if (2 * m + 1 < nlive) *reinterpret_cast<float2*>(p) = o;
    else *p = o.x;
  }
}

// Energy of every interior trace over its first nz samples, summed in order in float
// (src/fftgrid.cpp:2360-2371); nzero[l] counts the traces of angle l with zero energy (the
// only ones a zero threshold flags).
__global__ void k_trace_energy(const __grid_constant__ ThickParams P, float* energy, int* nzero) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, l = blockIdx.z;
  if (i >= P.nx) return;
  const float* g = P.grid[l] + (size_t)j * P.rnxp + i;
  const size_t kstride = (size_t)P.nyp * P.rnxp;
  float e = 0.f;
  for (int k = 0; k < P.nz; k++) {
    const float v = g[(size_t)k * kstride];
    e = __fadd_rn(e, __fmul_rn(v, v));
  }
  energy[((size_t)l * P.ny + j) * P.nx + i] = e;
  if (e == 0.f) atomicAdd(nzero + l, 1);
}

// interpolateTrace (src/fftgrid.cpp:2440-2480) for a list of independent operations: the
// target trace becomes the mean of its listed neighbours (left, right, up, down order).
__global__ void k_trace_interp(float* g, int rnxp, int nyp, int nzp, int nx, const TraceOp* ops) {
  const TraceOp op = ops[blockIdx.x];
  const size_t kstride = (size_t)nyp * rnxp;
  for (int k = blockIdx.y * blockDim.x + threadIdx.x; k < nzp; k += gridDim.y * blockDim.x) {
    float s = 0.f;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int n = op.nb[q];
      if (n >= 0) s = __fadd_rn(s, g[(size_t)k * kstride + (size_t)(n / nx) * rnxp + n % nx]);
    }
    g[(size_t)k * kstride + (size_t)(op.t / nx) * rnxp + op.t % nx] = __fdiv_rn(s, (float)op.nt);
  }
}

// extrapolateSeismic (src/fftgrid.cpp:2484-2516): every voxel of a trace outside the box
// of good traces takes the value of its mirror trace (getFillNumber, clamped into the box)
// times (max(1 - dx^2 - dy^2 - dz^2, 0))^3 of the distances to the boundary.  The mirror
// traces lie inside the box, which this kernel never writes.
// The launch covers only traces outside the box: rows0 = 1 takes the rows j < jmin and
// j > jmax (all i); rows0 = 0 the columns i < imin and i > imax of the rows inside.
__global__ void k_extrapolate(const __grid_constant__ ThickParams P, int l, int imin, int imax, int jmin, int jmax,
                              int rows0) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, k = blockIdx.z;
  int i, j;
  if (rows0) {
    i = x;
    j = y < jmin ? y : jmax + 1 + (y - jmin);
  } else {
    i = x < imin ? x : imax + 1 + (x - imin);
    j = jmin + y;
  }
  if (i >= P.nxp || j >= P.nyp) return;
  int ri = __ldg(P.fillx + i), rj = __ldg(P.filly + j);
  ri = ri < imin ? imin : (ri > imax ? imax : ri);
  rj = rj < jmin ? jmin : (rj > jmax ? jmax : rj);
  float* g = P.grid[l] + (size_t)k * P.nyp * P.rnxp;
  const float v = g[(size_t)rj * P.rnxp + ri];
  const float dx = __ldg(P.distx + i), dy = __ldg(P.disty + j), dz = __ldg(P.distz + k);
  double t = 1.0 - (double)__fmul_rn(dx, dx);
  t -= (double)__fmul_rn(dy, dy);
  t -= (double)__fmul_rn(dz, dz);
  t = t > 0.0 ? t : 0.0;
  const float mult = (float)(t * t * t);
  g[(size_t)j * P.rnxp + i] = __fmul_rn(mult, v);
}

// NRLib::RegularSurface<float>::GetZ (libs/nrlib/surface/regularsurface.hpp:367-394 with
// GetCorners :670-703, FindGeneralIndex :640-644, CellRelX/Y :851-863, GetBilinearZ :328-337
// and GetBilinearZMissingCorners :340-363; missing value -999) of a surface of ni x nj nodes
// (i + ni j) with origin (x0, y0) and spacing (dx, dy), in double as NRLib forms it.
__device__ float surface_z(const float* z, int ni, int nj, double x0, double y0, double dx, double dy,
                           double x, double y) {
  const float miss = -999.0f;
  const double fx = __ddiv_rn(x - x0, dx), fy = __ddiv_rn(y - y0, dy);
  const int i = (int)floor(fx), j = (int)floor(fy);
  float c[4] = {miss, miss, miss, miss};
  if (i + 1 >= 0 && i < ni && j + 1 >= 0 && j < nj) {
    if (i >= 0 && j >= 0) c[0] = z[i + (size_t)ni * j];
    if (i + 1 < ni && j >= 0) c[1] = z[i + 1 + (size_t)ni * j];
    if (i >= 0 && j + 1 < nj) c[2] = z[i + (size_t)ni * (j + 1)];
    if (i + 1 < ni && j + 1 < nj) c[3] = z[i + 1 + (size_t)ni * (j + 1)];
  }
  int nmiss = 0;
  for (int q = 0; q < 4; q++) nmiss += c[q] == miss;
  if (nmiss == 4) return miss;
  const double u = fx - trunc(fx), v = fy - trunc(fy);
  if (nmiss == 0) {
    const float a = c[0], b = __fsub_rn(c[1], a), cc = __fsub_rn(c[2], a);
    const float d = __fsub_rn(__fsub_rn(__fsub_rn(c[3], a), b), cc);
    const double r = __dadd_rn(__dadd_rn(__dadd_rn((double)a, __dmul_rn((double)b, u)), __dmul_rn((double)cc, v)),
                               __dmul_rn(__dmul_rn((double)d, u), v));
    return (float)r;
  }
  const double w[4] = {__dmul_rn(1.0 - u, 1.0 - v), __dmul_rn(u, 1.0 - v), __dmul_rn(1.0 - u, v), __dmul_rn(u, v)};
  double sum = 0.0, sw = 0.0;
  for (int q = 0; q < 4; q++)
    if (c[q] != miss) {
      sum = __dadd_rn(sum, __dmul_rn(w[q], (double)c[q]));
      sw = __dadd_rn(sw, w[q]);
    }
  if (sw == 0.0) return miss;
  return (float)__ddiv_rn(sum, sw);
}

// One thread per (unpadded trace, angle): Wavelet3D::getLocalStretch and
// createLocalWavelet1D (src/wavelet3D.cpp:328-373) with findPhi / findPsi (:819-851) and
// dipAdjustWavelet (:452-459).  The reference's float calls (atan and cos of float
// arguments) are taken as the double function rounded to float.  Then the norm^2 of the
// adjusted wavelet (Wavelet::findNorm, src/wavelet.cpp:882-900, by Parseval over the half
// spectrum in double) and gamma = 1 / findNormWithinFrequencyBand (:903-925) of the normalised
// errorSmooth3 table times the same dip factors.
__global__ void k_wavelet3d_fill(const __grid_constant__ Wavelet3DFill F) {
  const int l = blockIdx.y;
  const size_t nxy = (size_t)F.nx * F.ny;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nxy) return;
  const float gx = F.gx ? F.gx[t] : 0.f, gy = F.gy ? F.gy[t] : 0.f;
  const double pi = 3.14159265358979323846;
  double phi;
  const double eps = 0.001;
  if (gx > eps && gy >= 0.f) phi = (double)(float)atan((double)__fdiv_rn(gy, gx));
  else if (gx > eps && gy < 0.f) phi = __dadd_rn(2.0 * pi, (double)(float)atan((double)__fdiv_rn(gy, gx)));
  else if (gx < -eps) phi = __dadd_rn(pi, (double)(float)atan((double)__fdiv_rn(gy, gx)));
  else if (gy >= 0.f) phi = 0.5 * pi;
  else phi = 1.5 * pi;
  const float r = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy)), 1.f));
  const double psi = r > 1.f ? acos(__ddiv_rn(1.0, (double)r)) : 0.0;
  const double cth = (double)(float)cos((double)F.theta[l]);
  const double cpsi = __dmul_rn(cos(psi), cth);
  const double xd = __ddiv_rn(__dmul_rn(phi, 180.0), pi), yd = __ddiv_rn(__dmul_rn(psi, 180.0), pi);
  const size_t nij = (size_t)F.ni * F.nj;
  const float a1 = surface_z(F.alpha1 + l * nij, F.ni, F.nj, F.x0, F.y0, F.dx, F.dy, xd, yd);
  const float H = F.halpha ? surface_z(F.halpha + l * nij, F.ni, F.nj, F.x0, F.y0, F.dx, F.dy, xd, yd) : 0.f;
  const double mult = __dmul_rn((double)a1, cpsi);
  const int cn = F.cnzp;
  const float2* wa = F.wamp + (size_t)l * cn;
  double n2 = 0.0;
  for (int k = 0; k < cn; k++) {
    const float f = dip_factor(F.den, k, mult, H);
    const float2 c = __ldg(wa + k);
    const double cr = (double)__fmul_rn(c.x, f), ci = (double)__fmul_rn(c.y, f);
    const double wk = (k == 0 || (k == cn - 1 && !(F.nzp & 1))) ? 1.0 : 2.0;
    n2 = __dadd_rn(n2, __dmul_rn(wk, __dadd_rn(__dmul_rn(cr, cr), __dmul_rn(ci, ci))));
  }
  const float norm = (float)sqrt(__ddiv_rn(n2, (double)F.nzp));
  float gam = 1.f;
  if (F.es3) {
    const double fac = __ddiv_rn(1.0, (double)F.nzp);
    double e2 = 0.0;
    float e0 = 0.f;
    for (int k = F.loI; k < F.hiI; k++) {
      const float f = dip_factor(F.den, k, mult, H);
      const float2 c = k < cn - 1 ? __ldg(F.es3 + (size_t)l * cn + k) : F.es3_last[l];
      const float er = __fmul_rn(c.x, f), ei = __fmul_rn(c.y, f);
      const float p = __fadd_rn(__fmul_rn(er, er), __fmul_rn(ei, ei));
      if (k == 0) e0 = p;
      e2 = __dadd_rn(e2, __dmul_rn(2.0 * fac, (double)p));
    }
    if (F.loI == 0) e2 = __dsub_rn(e2, __dmul_rn(fac, (double)e0));
    gam = __fdiv_rn(1.f, (float)sqrt(e2));
  }
  F.mult[l * nxy + t] = mult;
  F.par[l * nxy + t] = make_float4(H, (float)cpsi, __fmul_rn(norm, norm), gam);
}

}  // namespace

size_t thick_smem_bytes(int W, int nzp) { return sizeof(float2) * ((size_t)nzp + 2 * (size_t)W * nzp); }

int thick_tile_width(int nzp) {
  for (int W = 16; W >= 1; W /= 2)
    if (thick_smem_bytes(W, nzp) <= 100 * 1024) return W;
  return 0;
}

cudaError_t launch_thick_divide(const ThickParams& P, int nth, cudaStream_t st, int* nlaunch) {
  if (P.W < 1 || P.W > 32 || (P.W & (P.W - 1)) || (1 << P.logW) != P.W) return cudaErrorInvalidValue;
  const size_t smem = thick_smem_bytes(P.W, P.nzp);
  const bool local = P.mode == 0 && (P.wshift || P.w3_mult);
  auto* k = local ? k_thick_divide<true> : k_thick_divide<false>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)P.nIT, (unsigned)(P.mode == 1 ? P.ny : P.nyp), (unsigned)nth);
  k<<<grid, 256, smem, st>>>(P);
  if (nlaunch) (*nlaunch)++;
  return cudaGetLastError();
}

cudaError_t launch_trace_energy(const ThickParams& P, int nth, float* energy, int* nzero, cudaStream_t st,
                                int* nlaunch) {
  cudaError_t e = cudaMemsetAsync(nzero, 0, sizeof(int) * nth, st);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)((P.nx + 127) / 128), (unsigned)P.ny, (unsigned)nth);
  k_trace_energy<<<grid, 128, 0, st>>>(P, energy, nzero);
  if (nlaunch) (*nlaunch)++;
  return cudaGetLastError();
}

cudaError_t launch_trace_interp(float* g, int rnxp, int nyp, int nzp, int nx, const TraceOp* ops, int nops,
                                cudaStream_t st, int* nlaunch) {
  if (nops <= 0) return cudaSuccess;
  dim3 grid((unsigned)nops, (unsigned)((nzp + 255) / 256));
  k_trace_interp<<<grid, 256, 0, st>>>(g, rnxp, nyp, nzp, nx, ops);
  if (nlaunch) (*nlaunch)++;
  return cudaGetLastError();
}

cudaError_t launch_wavelet3d_fill(const Wavelet3DFill& F, int nth, cudaStream_t st, int* nlaunch) {
  const size_t nxy = (size_t)F.nx * F.ny;
  if (nxy == 0 || nth < 1 || nth > kMaxTheta) return cudaErrorInvalidValue;
  dim3 grid((unsigned)((nxy + 127) / 128), (unsigned)nth);
  k_wavelet3d_fill<<<grid, 128, 0, st>>>(F);
  if (nlaunch) (*nlaunch)++;
  return cudaGetLastError();
}

cudaError_t launch_extrapolate(const ThickParams& P, int l, const int box[4], cudaStream_t st, int* nlaunch) {
  const int imin = box[0], imax = box[1], jmin = box[2], jmax = box[3];
  const int nrows = jmin + (P.nyp - 1 - jmax);         // rows outside the box
  const int ncols = imin + (P.nxp - 1 - imax);         // columns outside, rows inside
  if (nrows > 0) {
    dim3 grid((unsigned)((P.nxp + 127) / 128), (unsigned)nrows, (unsigned)P.nzp);
    k_extrapolate<<<grid, 128, 0, st>>>(P, l, imin, imax, jmin, jmax, 1);
    if (nlaunch) (*nlaunch)++;
  }
  if (ncols > 0) {
    const int T = std::min(128, (ncols + 31) / 32 * 32);
    dim3 grid((unsigned)((ncols + T - 1) / T), (unsigned)(jmax - jmin + 1), (unsigned)P.nzp);
    k_extrapolate<<<grid, T, 0, st>>>(P, l, imin, imax, jmin, jmax, 0);
    if (nlaunch) (*nlaunch)++;
  }
  return cudaGetLastError();
}

// ------------------------------------------------------------------ host side

// FFTGrid::getDistToBoundary (src/fftgrid.cpp:1158-1197) for 0 <= i < np.
float dist_to_boundary(int i, int n, int np) {
  if (i < n) return 0.f;
  const float taper = static_cast<float>(std::min(n, np - n) / 2.1);
  const int below = np - i, above = i - (n - 1);
  return above < below ? static_cast<float>(above) / taper : static_cast<float>(below) / taper;
}

// FFTGrid::getFillNumber (src/fftgrid.cpp:1103-1141) for 0 <= i < np.
int fill_number(int i, int n, int np) {
  if (i < n) return i;
  const int below = np - i - 1, above = i - n + 1;
  return above < below ? std::max(n - above, n / 2) : std::min(below, n / 2);
}

// The control flow of FFTGrid::interpolateSeismic (src/fftgrid.cpp:2349-2437) and
// interpolateTrace (:2440-2480) on the energy map of one angle: which trace is replaced
// by the mean of which neighbours, in the reference's order.  It depends on the flags
// only, never on the trace values, so it is planned here and executed on the device.  Each
// operation gets a level one above the highest level among the operations that produced
// its neighbours; operations of one level are independent (every trace is written at most
// once, and only traces with even flags -- good or already interpolated -- are read).
// Returns the operations grouped by level (level_start[L] .. level_start[L+1]) and the
// box of good traces {imin, imax, jmin, jmax}.
void plan_trace_interpolation(const float* energy, int nx, int ny, float threshold, std::vector<TraceOp>& ops,
                              std::vector<int>& level_start, int box[4]) {
  const int n = nx * ny;
  std::vector<short> flags(n);
  float total = 0.f;
  for (int q = 0; q < n; q++) total += energy[q];
  const float limit = threshold * total / float(n);
  int imin = nx, imax = 0, jmin = ny, jmax = 0, flag = 0;
  for (int j = 0, q = 0; j < ny; j++)
    for (int i = 0; i < nx; i++, q++) {
      const int cur = energy[q] <= limit ? 1 : 0;
      flags[q] = (short)(flag + cur);
      if (cur == 1) {
        flag = 2;
      } else {
        imin = std::min(imin, i);
        imax = std::max(imax, i);
        jmin = std::min(jmin, j);
        jmax = std::max(jmax, j);
      }
    }
  std::vector<int> level(n, 0);
  std::vector<TraceOp> raw;
  auto interp = [&](int index, int i, int j) -> int {
    const bool left = i > 0 && flags[index - 1] % 2 == 0;
    const bool right = i < nx - 1 && flags[index + 1] % 2 == 0;
    const bool up = j > 0 && flags[index - nx] % 2 == 0;
    const bool down = j < ny - 1 && flags[index + nx] % 2 == 0;
    const int nt = (int)left + (int)right + (int)up + (int)down;
    if (nt > 1) {
      TraceOp op;
      op.t = index;
      op.nb[0] = left ? index - 1 : -1;
      op.nb[1] = right ? index + 1 : -1;
      op.nb[2] = up ? index - nx : -1;
      op.nb[3] = down ? index + nx : -1;
      op.nt = nt;
      int lv = 0;
      for (int q = 0; q < 4; q++)
        if (op.nb[q] >= 0) lv = std::max(lv, level[op.nb[q]]);
      level[index] = lv + 1;
      raw.push_back(op);
      flags[index]--;
    }
    return flags[index];
  };
  for (int j = 0, cur = 0; j < ny; j++)
    for (int i = 0; i < nx; i++, cur++) {
      if (flags[cur] % 2 != 1) continue;
      if (interp(cur, i, j) % 2 != 0) continue;
      int index = cur - 1;
      while (index >= 0 && flags[index] > 1) {
        if (flags[index] % 2 == 1) interp(index, index % nx, index / nx);
        index--;
      }
      if (index < 0) index = 0;
      index++;
      while (index <= cur && flags[index - 1] == 0) {
        if (flags[index] > 1) flags[index] -= 2;
        index++;
      }
    }
  int maxl = 0;
  for (const TraceOp& op : raw) maxl = std::max(maxl, level[op.t]);
  level_start.assign(maxl + 2, 0);
  for (const TraceOp& op : raw) level_start[level[op.t] + 1]++;
  for (int L = 1; L < (int)level_start.size(); L++) level_start[L] += level_start[L - 1];
  ops.assign(raw.size(), TraceOp{});
  std::vector<int> fillp(level_start.begin(), level_start.end());
  for (const TraceOp& op : raw) ops[fillp[level[op.t]]++] = op;
  box[0] = imin;
  box[1] = imax;
  box[2] = jmin;
  box[3] = jmax;
}

}  // namespace crava
