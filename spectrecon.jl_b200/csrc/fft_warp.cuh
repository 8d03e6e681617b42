// fft_warp.cuh -- one-warp, shared-memory, in-place complex FFT (sm_100a).
//
// Replaces the FFTW plans of PlanPSF (src/plan-psf.jl:64-65, FFTW.jl compat
// "1") for the padded plane sizes of the projector: power-of-two lengths
// 1..SPECT_TW_N.  Algorithm: Stockham auto-sort (natural-order output) with
// one radix-2 stage when log2(n) is odd, then radix-4 stages.  Each stage
// loads all of the warp's butterfly inputs into registers, __syncwarp(),
// then stores the outputs in place, so one warp owns one transform and no
// block-level barrier is needed.  Twiddles come from a shared-memory table
// tw[m] = exp(-2 pi i m / SPECT_TW_N) computed on the host in double.
// Forward: X[k] = sum_m x[m] exp(-2 pi i k m / n); inverse uses +i; neither
// scales (the 1/(Npx*Npz) of the reference's ifft is folded into the PSF
// spectrum).
#pragma once
#include <cuda_runtime.h>

#define SPECT_TW_LOG 9
#define SPECT_TW_N 512
#define SPECT_FFT_MAXE (SPECT_TW_N / 32)

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// In-place transform of x[0..n) (shared memory owned by the calling warp).
template <bool INV>
__device__ __forceinline__ void warp_fft(float2* x, int n, int logn, const float2* __restrict__ tw, int lane) {
  int Ns = 1;
  if (logn & 1) {  // radix-2 stage, Ns = 1: y[2j + r] = x[j] +- x[j + n/2]
    const int nb = n >> 1;
    float2 a[SPECT_FFT_MAXE / 2], b[SPECT_FFT_MAXE / 2];
#pragma unroll
    for (int t = 0; t < SPECT_FFT_MAXE / 2; ++t) {
      int j = lane + 32 * t;
      if (j < nb) {
        a[t] = x[j];
        b[t] = x[j + nb];
      }
    }
    __syncwarp();
#pragma unroll
    for (int t = 0; t < SPECT_FFT_MAXE / 2; ++t) {
      int j = lane + 32 * t;
      if (j < nb) {
        x[2 * j] = cadd(a[t], b[t]);
        x[2 * j + 1] = csub(a[t], b[t]);
      }
    }
    __syncwarp();
    Ns = 2;
  }
  const int q = n >> 2;
  while (Ns < n) {  // radix-4 stage
    float2 v[SPECT_FFT_MAXE / 4][4];
#pragma unroll
    for (int t = 0; t < SPECT_FFT_MAXE / 4; ++t) {
      int j = lane + 32 * t;
      if (j < q) {
#pragma unroll
        for (int r = 0; r < 4; ++r) v[t][r] = x[j + r * q];
      }
    }
    __syncwarp();
    const int step = SPECT_TW_N / (4 * Ns);
#pragma unroll
    for (int t = 0; t < SPECT_FFT_MAXE / 4; ++t) {
      int j = lane + 32 * t;
      if (j < q) {
        int k = j & (Ns - 1);
        float2 w1 = tw[k * step], w2 = tw[2 * k * step], w3 = tw[3 * k * step];
        if (INV) {
          w1.y = -w1.y;
          w2.y = -w2.y;
          w3.y = -w3.y;
        }
        float2 v0 = v[t][0], v1 = cmul(v[t][1], w1), v2 = cmul(v[t][2], w2), v3 = cmul(v[t][3], w3);
        float2 s02 = cadd(v0, v2), d02 = csub(v0, v2), s13 = cadd(v1, v3), d13 = csub(v1, v3);
        // forward: y1 = d02 - i d13, y3 = d02 + i d13 ; inverse swaps the sign of i
        float2 id13 = make_float2(-d13.y, d13.x);  // i * d13
        float2 y1 = INV ? cadd(d02, id13) : csub(d02, id13);
        float2 y3 = INV ? csub(d02, id13) : cadd(d02, id13);
        int dst = (j - k) * 4 + k;
        x[dst] = cadd(s02, s13);
        x[dst + Ns] = y1;
        x[dst + 2 * Ns] = csub(s02, s13);
        x[dst + 3 * Ns] = y3;
      }
    }
    __syncwarp();
    Ns <<= 2;
  }
}
