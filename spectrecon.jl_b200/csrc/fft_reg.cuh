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
//   tw32[kb*32 + l]   = W_32^((l & 3) kb)            (256-point x transforms)
//   xpair[l]          = (baseA, fA, baseB, fB)        (256-point x transforms)
//   xscr              = per-warp transpose scratch, kXScr float2 per warp
struct FftTables {
  const float4* cross;
  const float2* rx;
  const float2* rz;
  const float2* base;
  const float2* tw32;
  const int4* xpair;
  float2* xscr;
};

constexpr int kXScr = 288;        // float2 per warp: 8 rows of 36 (first transpose)
constexpr int kConvWarpsMax = 16; // warps of the convolution kernels

__host__ __device__ constexpr int fft_x256_bytes(int RX) {
  return RX == 8 ? 8 * 32 * 8 + 32 * 16 + kConvWarpsMax * kXScr * 8 : 0;
}

__host__ __device__ constexpr int fft_tables_bytes(int RX, int RZ) {
  return SPECT_TW_N * 8 + 5 * 32 * 16 + (RX + RZ) * 32 * 8 + fft_x256_bytes(RX);
}

// ---- 256-point x transform (R = 8): the 32-point DFT across the lanes is
// split as 32 = 8 x 4 and done in registers between two shared-memory
// transposes, instead of five shuffle stages.
//   forward: lane l, register r holds x[l + 32 r].  8-point DFT over r and
//   twiddle W_256^(l k1) (as fft_fwd); transpose M[k1][l] (row stride 36) so
//   that lane 4 k1 + la holds M[k1][la + 4 lb], lb = 0..7; 8-point DFT over
//   lb, twiddle W_32^(la kb); transpose Z (address xz_addr) so that each lane
//   holds two (k1, kb) pairs A and B with la = 0..3; 4-point DFTs over la.
//   Register ka of pair A holds X[k1A + 8 kbA + 64 ka], register 4 + ka that
//   of pair B.  Pair B is the spectrum partner of pair A: X[-k] of register r
//   is register 7 - r of the same lane, except on lane 0, whose pairs (0, 0)
//   and (0, 4) are their own partners: register (4 - r) & 3 for r < 4 and
//   11 - r for r >= 4.  Both transposes are free of bank conflicts for 8-byte
//   accesses.
//   Lane l = 16 h + 4 q + i: pair A = (q, 4 h + i) for q = 1, 2, 3, (0, i) for
//   q = 0, h = 0 and (4, i) for q = 0, h = 1; pair B = (8 - k1A, 7 - kbA) when
//   k1A != 0, (0, 8 - kbA) when k1A == 0 < kbA, and (0, 4) for (0, 0).
__host__ __device__ constexpr int xz_addr(int k1, int kb, int la) { return 4 * (k1 + 8 * kb) + (la ^ (kb & 3)); }

__host__ __device__ inline void x256_pairs(int l, int& k1A, int& kbA, int& k1B, int& kbB) {
  const int h = l >> 4, q = (l >> 2) & 3, i = l & 3;
  k1A = q ? q : 4 * h;
  kbA = q ? 4 * h + i : i;
  if (k1A != 0) {
    k1B = 8 - k1A;
    kbB = 7 - kbA;
  } else {
    k1B = 0;
    kbB = kbA ? 8 - kbA : 4;
  }
}

// frequency index held by lane l, register r of a 256-point x transform
__host__ __device__ inline int x256_freq(int l, int r) {
  int k1A, kbA, k1B, kbB;
  x256_pairs(l, k1A, kbA, k1B, kbB);
  return r < 4 ? k1A + 8 * kbA + 64 * r : k1B + 8 * kbB + 64 * (r - 4);
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
  T.tw32 = nullptr;
  T.xpair = nullptr;
  T.xscr = nullptr;
  if (RX == 8) {
    float2* tw32 = rz + RZ * 32;
    int4* xpair = reinterpret_cast<int4*>(tw32 + 8 * 32);
    for (int k = threadIdx.x; k < 8 * 32; k += blockDim.x) {
      const int kb = k >> 5, l = k & 31;
      tw32[k] = tw_global[(((l & 3) * kb) << (SPECT_TW_LOG - 5)) & (SPECT_TW_N - 1)];
    }
    for (int l = threadIdx.x; l < 32; l += blockDim.x) {
      int k1A, kbA, k1B, kbB;
      x256_pairs(l, k1A, kbA, k1B, kbB);
      xpair[l] = make_int4(4 * (k1A + 8 * kbA), kbA & 3, 4 * (k1B + 8 * kbB), kbB & 3);
    }
    T.tw32 = tw32;
    T.xpair = xpair;
    T.xscr = reinterpret_cast<float2*>(xpair + 32);
  }
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

template <int R>
__device__ __forceinline__ void reg_dft_at(float2 (&v)[8], int o, const float2* __restrict__ base) {
  float2 t[R];
#pragma unroll
  for (int k = 0; k < R; ++k) t[k] = v[o + k];
  reg_dft<R>(t, base);
#pragma unroll
  for (int k = 0; k < R; ++k) v[o + k] = t[k];
}

// 256-point forward x transform (see the layout above); w = this warp's
// transpose scratch, rtw = FftTables::rx + lane
__device__ __forceinline__ void fftx256_fwd(float2 (&v)[8], int lane, const FftTables& T,
                                            const float2* __restrict__ rtw, float2* w) {
  reg_dft<8>(v, T.base);
#pragma unroll
  for (int k1 = 1; k1 < 8; ++k1) v[k1] = cmul(v[k1], rtw[k1 * 32]);
  __syncwarp();
#pragma unroll
  for (int k1 = 0; k1 < 8; ++k1) w[k1 * 36 + lane] = v[k1];
  __syncwarp();
  const int k1 = lane >> 2, la = lane & 3;
#pragma unroll
  for (int lb = 0; lb < 8; ++lb) v[lb] = w[k1 * 36 + la + 4 * lb];
  reg_dft<8>(v, T.base);
#pragma unroll
  for (int kb = 1; kb < 8; ++kb) v[kb] = cmul(v[kb], T.tw32[kb * 32 + lane]);
  __syncwarp();
#pragma unroll
  for (int kb = 0; kb < 8; ++kb) w[xz_addr(k1, kb, la)] = v[kb];
  __syncwarp();
  const int4 pr = T.xpair[lane];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    v[a] = w[pr.x + (a ^ pr.y)];
    v[4 + a] = w[pr.z + (a ^ pr.w)];
  }
  reg_dft_at<4>(v, 0, T.base);
  reg_dft_at<4>(v, 4, T.base);
}

// inverse of fftx256_fwd (unscaled: returns 256 x[l + 32 r] in register r)
__device__ __forceinline__ void fftx256_inv(float2 (&v)[8], int lane, const FftTables& T,
                                            const float2* __restrict__ rtw, float2* w) {
  // conj(IDFT(y)) = DFT(conj(y)): carry the conjugate through the stages
#pragma unroll
  for (int r = 0; r < 8; ++r) v[r] = cconj(v[r]);
  reg_dft_at<4>(v, 0, T.base);
  reg_dft_at<4>(v, 4, T.base);
  const int4 pr = T.xpair[lane];
  __syncwarp();
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    w[pr.x + (a ^ pr.y)] = v[a];
    w[pr.z + (a ^ pr.w)] = v[4 + a];
  }
  __syncwarp();
  const int k1 = lane >> 2, la = lane & 3;
#pragma unroll
  for (int kb = 0; kb < 8; ++kb) v[kb] = w[xz_addr(k1, kb, la)];
#pragma unroll
  for (int kb = 1; kb < 8; ++kb) v[kb] = cmul(v[kb], T.tw32[kb * 32 + lane]);
  reg_dft<8>(v, T.base);
  __syncwarp();
#pragma unroll
  for (int lb = 0; lb < 8; ++lb) w[k1 * 36 + la + 4 * lb] = v[lb];
  __syncwarp();
#pragma unroll
  for (int q = 0; q < 8; ++q) v[q] = w[q * 36 + lane];
#pragma unroll
  for (int q = 1; q < 8; ++q) v[q] = cmul(v[q], rtw[q * 32]);
  reg_dft<8>(v, T.base);
#pragma unroll
  for (int r = 0; r < 8; ++r) v[r] = cconj(v[r]);
}

// x transforms of the convolution kernels: 256 points through shared
// memory, other lengths by fft_fwd / fft_inv
template <int R>
__device__ __forceinline__ void fftx_fwd(float2 (&v)[R], int lc, int logC_rt, const FftTables& T,
                                         const float2* __restrict__ rtw, float2* w) {
  if constexpr (R == 8) fftx256_fwd(v, lc, T, rtw, w);
  else fft_fwd<R>(v, lc, logC_rt, T, rtw);
}
template <int R>
__device__ __forceinline__ void fftx_inv(float2 (&v)[R], int lc, int logC_rt, const FftTables& T,
                                         const float2* __restrict__ rtw, float2* w) {
  if constexpr (R == 8) fftx256_inv(v, lc, T, rtw, w);
  else fft_inv<R>(v, lc, logC_rt, T, rtw);
}
