// rot_one.cuh -- imrotate! / imrotate_adj! with interpmeth = :one on sm_100a:
// the 3-pass shear rotation of src/rotatez.jl:240-322 with the 1-D linear
// SparseInterpolator set up by linearinterp! (src/rotatez.jl:21-51).
//
// One CTA rotates one nx x nx slice on the zero-padded L x L grid
// (L = nx + 2*pad, pad = ceil(1 + nx*sqrt(2)/2 - nx/2), src/plan-rotate.jl:56),
// held in shared memory (or a per-CTA global slab when it does not fit) with
// leading dimension LS = L + 1 (odd: row lines are bank-conflict free).
// Element (a, b) (a along dim 1 = x, b along dim 2 = y) is W[a + LS*b].
// The 90-degree pre-rotation (rot_f90!) is folded into the load, its adjoint
// into the final read; each shear is done line by line through a per-warp
// line buffer.  Line parameters are computed in Float64 exactly as the
// reference does (positions in Float64, coefficients rounded to Float32).
#pragma once
#include <cuda_runtime.h>

namespace spect {

constexpr int kRot1Threads = 512;
constexpr int kRot1Warps = kRot1Threads / 32;

struct Rot1Geom {
  int nx, ny, nz, L, pad, LS;
};

// per view: mode 0 copy (theta == 0 mod 2pi), 1 rot_f90 only (theta close
// to m*pi/2), 2 rot_f90 + shears; tn = tan(phi/2), sn = -sin(phi),
// phi = theta - m*pi/2 (src/rotatez.jl:249-272)
struct Rot1View {
  double tn, sn;
  int m, mode;
};

// linearinterp!(A, s, e, len) for the line with 1-based index i; the output
// sample q (0-based) is  C_lo * x[J_lo(q)-1] + C_hi * x[J_hi(q)-1]
struct Line1 {
  float clo, chi;
  int caseA;  // e <= len: J = max(1, K - L + q (+1)); else J = min(L, F + q (+1))
  int K, F;
  __device__ __forceinline__ Line1(int i, double t, int L) {
    const double c = (L + 1) / 2.0;
    const double s = (i - c) * t + 1, e = (i - c) * t + L;
    const double dec = ceil(s) - s;
    clo = (float)dec;
    chi = (float)(1.0 - dec);
    caseA = e <= L;
    K = (int)ceil(e);
    F = (int)floor(s);
  }
  __device__ __forceinline__ int jlo(int q, int L) const {  // 1-based
    return caseA ? max(1, K - L + q) : min(L, F + q);
  }
  __device__ __forceinline__ int jhi(int q, int L) const {
    return caseA ? max(1, K - L + 1 + q) : min(L, F + q + 1);
  }
};

// y = A x on one line (x in the warp's line buffer, y to W with stride ws)
__device__ __forceinline__ void line_fwd(const Line1& P, const float* __restrict__ x, float* y, int ws, int L,
                                         int lane) {
  for (int q = lane; q < L; q += 32) {
    const float a = __fmul_rn(P.clo, x[P.jlo(q, L) - 1]);
    const float b = __fmul_rn(P.chi, x[P.jhi(q, L) - 1]);
    y[(size_t)q * ws] = __fadd_rn(a, b);
  }
}

// y = A' x on one line, as a gather: interior outputs have one q for each
// coefficient; the clamped edge output sums its q range in increasing q,
// lo before hi, like the reference's transposed scatter
__device__ __forceinline__ void line_adj(const Line1& P, const float* __restrict__ x, float* y, int ws, int L,
                                         int lane) {
  for (int j = lane + 1; j <= L; j += 32) {  // 1-based output index
    float acc = 0.f;
    const bool edge = P.caseA ? (j == 1) : (j == L);
    if (!edge) {
      // J_lo(q) = j and J_hi(q') = j for exactly one q, q' each (if in range)
      int ql, qh;
      if (P.caseA) {
        ql = j + L - P.K;
        qh = ql - 1;
      } else {
        ql = j - P.F;
        qh = ql - 1;
      }
      // increasing q: the hi term (q' = q - 1) comes first
      if (qh >= 0 && qh < L) acc = __fadd_rn(acc, __fmul_rn(P.chi, x[qh]));
      if (ql >= 0 && ql < L) acc = __fadd_rn(acc, __fmul_rn(P.clo, x[ql]));
    } else {
      for (int q = 0; q < L; ++q) {
        if (P.jlo(q, L) == j) acc = __fadd_rn(acc, __fmul_rn(P.clo, x[q]));
        if (P.jhi(q, L) == j) acc = __fadd_rn(acc, __fmul_rn(P.chi, x[q]));
      }
    }
    y[(size_t)(j - 1) * ws] = acc;
  }
}

// one shear pass over all lines of W.  ALONG_X: lines are columns (fixed b,
// contiguous); else rows (fixed a, stride LS).  ADJ selects A'.
template <bool ALONG_X, bool ADJ>
__device__ __forceinline__ void shear_pass(float* W, float* linebuf, const Rot1Geom& G, double t, int warp,
                                           int lane) {
  const int L = G.L, LS = G.LS;
  for (int ln = warp; ln < L; ln += kRot1Warps) {
    float* line = ALONG_X ? W + (size_t)ln * LS : W + ln;
    const int ws = ALONG_X ? 1 : LS;
    for (int q = lane; q < L; q += 32) linebuf[q] = line[(size_t)q * ws];
    __syncwarp();
    const Line1 P(ln + 1, t, L);
    if (ADJ) line_adj(P, linebuf, line, ws, L, lane);
    else line_fwd(P, linebuf, line, ws, L, lane);
    __syncwarp();
  }
}

// position in W of padded element (a, b) after rot_f90! by m
// (rotl90 m=1, rot180 m=2, rotr90 m=3; src/rotatez.jl:155-210)
__device__ __forceinline__ int rot90_pos(int a, int b, int m, int L, int LS) {
  switch (m) {
    case 1: return (L - 1 - b) + LS * a;
    case 2: return (L - 1 - a) + LS * (L - 1 - b);
    case 3: return b + LS * (L - 1 - a);
  }
  return a + LS * b;
}
// element (a, b) of rot_f90_adj!(W, m) (rotr90 m=1, rot180 m=2, rotl90 m=3)
__device__ __forceinline__ int rot90adj_src(int a, int b, int m, int L, int LS) {
  switch (m) {
    case 1: return (L - 1 - b) + LS * a;
    case 2: return (L - 1 - a) + LS * (L - 1 - b);
    case 3: return b + LS * (L - 1 - a);
  }
  return a + LS * b;
}

// Forward :one rotation of slices: grid (nz, <= nv), slots strided over
// blockIdx.y; out[slot][z][y][x] = imrotate!(src[z], theta(view(slot))).
// src is one volume [nz][ny][nx] (src_per_slot = 0) or per-slot volumes.
__global__ void __launch_bounds__(kRot1Threads, 1) k_rot1_fwd(Rot1Geom G, const float* __restrict__ src,
                                                               int src_per_slot, const Rot1View* __restrict__ views,
                                                               const int* __restrict__ vidx, int nv,
                                                               float* __restrict__ out, int use_smem,
                                                               float* __restrict__ gscr) {
  extern __shared__ float4 smem4[];
  const int nx = G.nx, L = G.L, LS = G.LS, pad = G.pad;
  const int z = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t slice = (size_t)nx * nx;
  float* W;
  float* lines;
  const size_t wsz = (size_t)LS * L;
  if (use_smem) {
    W = reinterpret_cast<float*>(smem4);
    lines = W + wsz;
  } else {
    const size_t cta = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
    W = gscr + cta * (wsz + (size_t)kRot1Warps * L);
    lines = W + wsz;
  }
  float* linebuf = lines + (size_t)warp * L;
  for (int slot = blockIdx.y; slot < nv; slot += gridDim.y) {
    const float* in = src + ((src_per_slot ? (size_t)slot * G.nz : 0) + z) * slice;
    float* o = out + ((size_t)slot * G.nz + z) * slice;
    const Rot1View V = views[vidx[slot]];
    __syncthreads();
    if (V.mode == 0) {
      for (int k = threadIdx.x; k < (int)slice; k += blockDim.x) o[k] = in[k];
      continue;
    }
    for (size_t k = threadIdx.x; k < wsz; k += blockDim.x) W[k] = 0.f;
    __syncthreads();
    for (int k = threadIdx.x; k < (int)slice; k += blockDim.x) {
      const int j = k / nx, i = k - j * nx;
      W[rot90_pos(pad + i, pad + j, V.m, L, LS)] = in[k];
    }
    __syncthreads();
    if (V.mode == 2) {
      shear_pass<true, false>(W, linebuf, G, V.tn, warp, lane);
      __syncthreads();
      shear_pass<false, false>(W, linebuf, G, V.sn, warp, lane);
      __syncthreads();
      shear_pass<true, false>(W, linebuf, G, V.tn, warp, lane);
      __syncthreads();
    }
    for (int k = threadIdx.x; k < (int)slice; k += blockDim.x) {
      const int j = k / nx, i = k - j * nx;
      o[k] = W[(pad + i) + LS * (pad + j)];
    }
  }
}

// Adjoint :one rotation accumulated over views: grid (nz, nsplit);
// imgpart[split][z] (+)= sum over the split's slots of imrotate_adj!(S[slot][z]).
__global__ void __launch_bounds__(kRot1Threads, 1) k_rot1_adj(Rot1Geom G, const float* __restrict__ S,
                                                               const Rot1View* __restrict__ views,
                                                               const int* __restrict__ vidx, int nv,
                                                               float* __restrict__ imgpart, int accumulate,
                                                               int use_smem, float* __restrict__ gscr) {
  extern __shared__ float4 smem4[];
  const int nx = G.nx, L = G.L, LS = G.LS, pad = G.pad;
  const int z = blockIdx.x, split = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int slice = nx * nx;
  const size_t wsz = (size_t)LS * L;
  float *acc, *W, *lines;
  if (use_smem) {
    acc = reinterpret_cast<float*>(smem4);
    W = acc + slice;
    lines = W + wsz;
  } else {
    const size_t cta = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
    acc = gscr + cta * (slice + wsz + (size_t)kRot1Warps * L);
    W = acc + slice;
    lines = W + wsz;
  }
  float* linebuf = lines + (size_t)warp * L;
  float* outp = imgpart + ((size_t)split * G.nz + z) * slice;
  for (int k = threadIdx.x; k < slice; k += blockDim.x) acc[k] = accumulate ? outp[k] : 0.f;
  const int per = (nv + gridDim.y - 1) / gridDim.y;
  const int s0 = split * per, s1 = min(nv, s0 + per);
  for (int s = s0; s < s1; ++s) {
    const Rot1View V = views[vidx[s]];
    const float* in = S + ((size_t)s * G.nz + z) * slice;
    __syncthreads();
    if (V.mode == 0) {
      for (int k = threadIdx.x; k < slice; k += blockDim.x) acc[k] = __fadd_rn(acc[k], in[k]);
      continue;
    }
    for (size_t k = threadIdx.x; k < wsz; k += blockDim.x) W[k] = 0.f;
    __syncthreads();
    for (int k = threadIdx.x; k < slice; k += blockDim.x) {
      const int j = k / nx, i = k - j * nx;
      W[(pad + i) + LS * (pad + j)] = in[k];
    }
    __syncthreads();
    if (V.mode == 2) {
      shear_pass<true, true>(W, linebuf, G, V.tn, warp, lane);
      __syncthreads();
      shear_pass<false, true>(W, linebuf, G, V.sn, warp, lane);
      __syncthreads();
      shear_pass<true, true>(W, linebuf, G, V.tn, warp, lane);
      __syncthreads();
    }
    for (int k = threadIdx.x; k < slice; k += blockDim.x) {
      const int j = k / nx, i = k - j * nx;
      acc[k] = __fadd_rn(acc[k], W[rot90adj_src(pad + i, pad + j, V.m, L, LS)]);
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < slice; k += blockDim.x) outp[k] = acc[k];
}

// att[v][y][z][x] from the rotated mu-map Rm[v][z][y][x] by the depth scan
// (src/project.jl:103-113); grid-stride over (v, z, x)
__global__ void k_att_scan(const float* __restrict__ Rm, int nv, int nx, int ny, int nz, float dy,
                           float* __restrict__ att) {
  const size_t n = (size_t)nv * nz * nx;
  const float mdy = -dy;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(k % nx);
    const size_t r = k / nx;
    const int z = (int)(r % nz);
    const size_t v = r / nz;
    const float* m = Rm + ((v * nz + z) * ny) * nx + x;
    float* a = att + ((v * ny) * nz + z) * nx + x;
    float prefix = 0.f;
    for (int y = 0; y < ny; ++y) {
      const float mu = m[(size_t)y * nx];
      const float e = __fadd_rn(prefix, __fmul_rn(0.5f, mu));
      a[(size_t)y * nz * nx] = expf(__fmul_rn(e, mdy));
      prefix = __fadd_rn(prefix, mu);
    }
  }
}

// P[slot][y][z][x] = att[v][y][z][x] * R[slot][z][y][x]  (MUL_T = false), or
// S[slot][z][y][x] = att[v][y][z][x] * T[slot][y][z][x]   (MUL_T = true)
template <bool MUL_T>
__global__ void k_att_combine(const float* __restrict__ att, const float* __restrict__ in, const int* __restrict__ vidx,
                              int nv, int nx, int ny, int nz, float* __restrict__ out) {
  const size_t n = (size_t)nv * ny * nz * nx;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(k % nx);
    size_t r = k / nx;
    const int z = (int)(r % nz);
    r /= nz;
    const int y = (int)(r % ny);
    const size_t s = r / ny;
    const size_t yzx = (((size_t)vidx[s] * ny + y) * nz + z) * nx + x;     // att[v][y][z][x]
    const size_t syzx = ((s * ny + y) * nz + z) * nx + x;                   // [slot][y][z][x]
    const size_t szyx = ((s * nz + z) * ny + y) * nx + x;                   // [slot][z][y][x]
    if (MUL_T) out[szyx] = __fmul_rn(att[yzx], in[syzx]);
    else out[syzx] = __fmul_rn(in[szyx], att[yzx]);
  }
}

}  // namespace spect
