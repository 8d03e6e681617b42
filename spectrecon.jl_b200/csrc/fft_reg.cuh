// fft_reg.cuh -- register-resident warp FFT (sm_100a), the FFT engine of the
// projector's PSF convolution (replaces FFTW's plan_fft!/plan_ifft! of
// PlanPSF, src/plan-psf.jl:64-65).
//
// A length-N transform (N = R * C, C = min(32, N) lanes, R registers per
// lane, N a power of two <= SPECT_TW_N) is held by a group of C lanes; a warp
// runs 32 / C transforms side by side.  Lane l (0 <= l < C) starts with
// x[l + C r] in register r.
//   forward: R-point DFT in registers, twiddle W_N^(l k1), then a C-point DFT
//            across the lanes (radix-2 decimation in frequency, __shfl_xor_sync).
//            Lane l ends with X[k1 + R brev_C(l)] in register k1 ("scrambled"
//            order; brev_C reverses log2(C) bits).
//   inverse: consumes that scrambled order and returns natural order
//            (decimation in time across lanes, conjugate twiddles, inverse
//            R-point DFT): lane l ends with N * x[l + C r] in register r.
// Point-wise products with a spectrum therefore never need a reordering: the
// PSF spectra are stored in the same scrambled order at plan time.
// The spectrum partner X[-k] of register k1 lives in lane l ^ (C-1), register
// R - k1 (k1 > 0), or lane brev_C((C - brev_C(l)) mod C), register 0 (k1 == 0).
#pragma once
#include <cuda_runtime.h>

#define SPECT_TW_LOG 9
#define SPECT_TW_N 512

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

__host__ __device__ constexpr int brev_c(int x, int bits) {
  int r = 0;
  for (int b = 0; b < bits; ++b)
    if (x & (1 << b)) r |= 1 << (bits - 1 - b);
  return r;
}
__host__ __device__ constexpr int ilog2_c(int x) { return x <= 1 ? 0 : 1 + ilog2_c(x >> 1); }

__device__ __forceinline__ int brev_rt(int x, int bits) { return bits ? (__brev(x) >> (32 - bits)) : 0; }

__device__ __forceinline__ float2 shfl_xor2(float2 v, int m) {
  return make_float2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}
__device__ __forceinline__ float2 shfl2(float2 v, int src) {
  return make_float2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

// R-point forward DFT of the registers (natural order in and out).
// Radix-2 decimation in frequency, then a compile-time bit-reversal.
template <int R>
__device__ __forceinline__ void reg_dft(float2 (&v)[R], const float2* __restrict__ tw) {
#pragma unroll
  for (int half = R / 2; half >= 1; half >>= 1) {
#pragma unroll
    for (int b = 0; b < R; b += 2 * half) {
#pragma unroll
      for (int j = 0; j < half; ++j) {
        float2 a = v[b + j], c = v[b + j + half];
        v[b + j] = cadd(a, c);
        float2 d = csub(a, c);
        const int ti = j * (SPECT_TW_N / (2 * half));
        if (ti == 0) v[b + j + half] = d;
        else if (ti == SPECT_TW_N / 4) v[b + j + half] = make_float2(d.y, -d.x);  // * (-i)
        else v[b + j + half] = cmul(d, tw[ti]);
      }
    }
  }
  if (R > 2) {
    float2 t[R];
#pragma unroll
    for (int k = 0; k < R; ++k) t[k] = v[brev_c(k, ilog2_c(R))];
#pragma unroll
    for (int k = 0; k < R; ++k) v[k] = t[k];
  }
}

// forward transform; lc = lane within the C-lane group, logC = log2(C)
template <int R>
__device__ __forceinline__ void fft_fwd(float2 (&v)[R], int lc, int logC, int logN, const float2* __restrict__ tw) {
  reg_dft<R>(v, tw);
  if (R > 1) {
    const int sh = SPECT_TW_LOG - logN;
#pragma unroll
    for (int k1 = 1; k1 < R; ++k1) {
      v[k1] = cmul(v[k1], tw[((lc * k1) << sh) & (SPECT_TW_N - 1)]);
    }
  }
  // branch-free butterflies: lower lane a+b, upper lane (a-b) w, written
  // as (u + sg*v) * w_eff with sg = -1 and w_eff = w on the upper lane
  for (int s = logC - 1; s >= 0; --s) {
    const int m = 1 << s;
    const bool up = (lc & m) != 0;
    const float sg = up ? -1.f : 1.f;
    const float2 w = up ? tw[(lc & (m - 1)) << (SPECT_TW_LOG - s - 1)] : make_float2(1.f, 0.f);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      float2 u = shfl_xor2(v[r], m);
      float2 t = make_float2(fmaf(sg, v[r].x, u.x), fmaf(sg, v[r].y, u.y));
      v[r] = cmul(t, w);
    }
  }
}

// inverse transform (scrambled in, natural out, unscaled)
template <int R>
__device__ __forceinline__ void fft_inv(float2 (&v)[R], int lc, int logC, int logN, const float2* __restrict__ tw) {
  // inverse butterflies: the upper lane pre-multiplies by conj(w), then
  // lower = v + u, upper = u - v
  for (int s = 0; s < logC; ++s) {
    const int m = 1 << s;
    const bool up = (lc & m) != 0;
    const float sg = up ? -1.f : 1.f;
    float2 w = up ? tw[(lc & (m - 1)) << (SPECT_TW_LOG - s - 1)] : make_float2(1.f, 0.f);
    w.y = -w.y;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      float2 t = cmul(v[r], w);
      float2 u = shfl_xor2(t, m);
      v[r] = make_float2(fmaf(sg, t.x, u.x), fmaf(sg, t.y, u.y));
    }
  }
  if (R > 1) {
    const int sh = SPECT_TW_LOG - logN;
#pragma unroll
    for (int k1 = 1; k1 < R; ++k1) {
      v[k1] = cmulc(v[k1], tw[((lc * k1) << sh) & (SPECT_TW_N - 1)]);
    }
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = cconj(v[r]);
    reg_dft<R>(v, tw);
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = cconj(v[r]);
  }
}

// X[-k] for every register (see header); gbase = first lane of the group
template <int R>
__device__ __forceinline__ void spectrum_partner(const float2 (&v)[R], float2 (&p)[R], int lc, int logC, int gbase) {
  const int C = 1 << logC;
#pragma unroll
  for (int k1 = 1; k1 < R; ++k1) p[k1] = shfl_xor2(v[R - k1], C - 1);
  const int src = brev_rt((C - brev_rt(lc, logC)) & (C - 1), logC);
  p[0] = shfl2(v[0], gbase + src);
}
