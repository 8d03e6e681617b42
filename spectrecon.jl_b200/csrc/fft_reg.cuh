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
//
// For R >= 2 the lane count is 32 at compile time, so every stage loop is
// unrolled.  The lane-dependent twiddles come from small per-lane tables in
// shared memory built once per kernel (FftTables): no index arithmetic per
// transform.  Complex additions use the paired FP32 instructions of sm_100
// (__fadd2_rn / __ffma2_rn).
#pragma once
#include <cuda_runtime.h>

#define SPECT_TW_LOG 9
#define SPECT_TW_N 512

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }

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

// Shared-memory twiddle tables of one kernel.
//   cross[s*32 + l] = (w.x, w.y, sg, 0): cross-lane stage s (span 2^s) of lane
//                     l: the upper lane (bit s of l set) has sg = -1 and
//                     w = W_{2^(s+1)}^(l mod 2^s); the lower lane sg = +1, w = 1
//   rx[k1*32 + l]   = W_Npx^(l k1), rz[k1*32 + l] = W_Npz^(l k1)
//   base            = W_512^m, m < 512 (for the in-register DFTs)
struct FftTables {
  const float4* cross;
  const float2* rx;
  const float2* rz;
  const float2* base;
};

__host__ __device__ constexpr int fft_tables_bytes(int RX, int RZ) {
  return SPECT_TW_N * 8 + 5 * 32 * 16 + (RX + RZ) * 32 * 8;
}

// builds the tables in shared memory at `smem` (fft_tables_bytes(RX, RZ)
// bytes); call with all threads, then __syncthreads()
__device__ __forceinline__ FftTables build_fft_tables(float2* smem, const float2* __restrict__ tw_global, int RX,
                                                      int logNpx, int RZ, int logNpz) {
  FftTables T;
  float2* base = smem;
  float4* cross = reinterpret_cast<float4*>(base + SPECT_TW_N);
  float2* rx = reinterpret_cast<float2*>(cross + 5 * 32);
  float2* rz = rx + RX * 32;
  for (int k = threadIdx.x; k < SPECT_TW_N; k += blockDim.x) base[k] = tw_global[k];
  for (int k = threadIdx.x; k < 5 * 32; k += blockDim.x) {
    const int s = k >> 5, l = k & 31, m = 1 << s;
    const bool up = (l & m) != 0;
    const float2 w = up ? tw_global[(l & (m - 1)) << (SPECT_TW_LOG - s - 1)] : make_float2(1.f, 0.f);
    cross[k] = make_float4(w.x, w.y, up ? -1.f : 1.f, 0.f);
  }
  for (int k = threadIdx.x; k < RX * 32; k += blockDim.x) {
    const int k1 = k >> 5, l = k & 31;
    rx[k] = tw_global[((l * k1) << (SPECT_TW_LOG - logNpx)) & (SPECT_TW_N - 1)];
  }
  for (int k = threadIdx.x; k < RZ * 32; k += blockDim.x) {
    const int k1 = k >> 5, l = k & 31;
    rz[k] = tw_global[((l * k1) << (SPECT_TW_LOG - logNpz)) & (SPECT_TW_N - 1)];
  }
  T.cross = cross;
  T.rx = rx;
  T.rz = rz;
  T.base = base;
  return T;
}

// R-point forward DFT of the registers (natural order in and out).
// Radix-2 decimation in frequency, then a compile-time bit-reversal.
template <int R>
__device__ __forceinline__ void reg_dft(float2 (&v)[R], const float2* __restrict__ base) {
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
        else v[b + j + half] = cmul(d, base[ti]);
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

// forward transform.  lc = lane within the group; logC_rt used only when
// R == 1; rtw = this lane's register twiddles (FftTables::rx or rz, + lc)
template <int R>
__device__ __forceinline__ void fft_fwd(float2 (&v)[R], int lc, int logC_rt, const FftTables& T,
                                        const float2* __restrict__ rtw) {
  const int logC = (R > 1) ? 5 : logC_rt;
  reg_dft<R>(v, T.base);
#pragma unroll
  for (int k1 = 1; k1 < R; ++k1) v[k1] = cmul(v[k1], rtw[k1 * 32]);
  // branch-free butterflies: lower lane a+b, upper lane (a-b) w, written as
  // (u + sg*v) * w_eff with the per-lane (w_eff, sg) of the stage
#pragma unroll
  for (int s = 4; s >= 0; --s) {
    if (s < logC) {
      const float4 c = T.cross[s * 32 + lc];
      const float2 w = make_float2(c.x, c.y), sg = make_float2(c.z, c.z);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const float2 u = shfl_xor2(v[r], 1 << s);
        v[r] = cmul(__ffma2_rn(sg, v[r], u), w);
      }
    }
  }
}

// inverse transform (scrambled in, natural out, unscaled)
template <int R>
__device__ __forceinline__ void fft_inv(float2 (&v)[R], int lc, int logC_rt, const FftTables& T,
                                        const float2* __restrict__ rtw) {
  const int logC = (R > 1) ? 5 : logC_rt;
  // the upper lane pre-multiplies by conj(w), then lower = v + u, upper = u - v
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    if (s < logC) {
      const float4 c = T.cross[s * 32 + lc];
      const float2 w = make_float2(c.x, c.y), sg = make_float2(c.z, c.z);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const float2 t = cmulc(v[r], w);
        const float2 u = shfl_xor2(t, 1 << s);
        v[r] = __ffma2_rn(sg, t, u);
      }
    }
  }
  if (R > 1) {
#pragma unroll
    for (int k1 = 1; k1 < R; ++k1) v[k1] = cmulc(v[k1], rtw[k1 * 32]);
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = cconj(v[r]);
    reg_dft<R>(v, T.base);
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = cconj(v[r]);
  }
}
