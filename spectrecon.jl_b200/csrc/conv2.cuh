// conv2.cuh -- depth-dependent PSF convolution kernels (sm_100a), templated
// on the register counts RX = Npx/CX and RZ = Npz/CZ of the two FFT axes.
//
// Reference semantics: fft_conv! / fft_conv_adj! (src/fft_convolve.jl:33-130)
// on planes replicate-padded (adjoint: zero-padded then folded) to
// Npx x Npz = Power2(nx+px-1) x Power2(nz+pz-1) (src/helper.jl:8-12), with
// the depth sum of project! (src/project.jl:127-130).
//
// Data layout on chip, per CTA:
//   B[x][c]  (shared memory when it fits, else a per-CTA global slab), nx
//            rows of QS = Q+1 complex: the z-spectrum of each image row at the
//            Q = Npz/2 stored z-frequencies.  Column c holds kz = k1 +
//            RZ*brev(2*(c mod CZ/2)) with k1 = c / (CZ/2) (the scrambled order
//            of the z transform, even lanes), except column 0 which packs the
//            two real columns kz = 0 (.x) and kz = Npz/2 (.y).  The same
//            memory first holds the real plane, row x at floats [2*QS*x, +nz).
//   x-spectra live in registers in the scrambled order of fft_reg.cuh; the
//   plan stores the PSF spectra in exactly that order:
//     Hs[set][y][c][k1*CX + l]  = H(kx, kz(c)) / (Npx*Npz),  c = 1..Q-1
//     Hs[set][y][0][..] = (H(kx,0) + H(kx,Npz/2))/2, Hs[set][y][Q][..] = (H(kx,0) - H(kx,Npz/2))/2
//   so that for the packed column Y' = alpha*Y + beta*conj(Y(-kx)).
// Forward: the x-spectra of all planes of a depth chunk are multiplied by
// their PSF spectra and summed in registers (one inverse transform per chunk,
// not per plane).  Adjoint: the view spectrum is computed once (k_vspec2) and
// held in registers across the chunk.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fft_reg.cuh"
#include "bulk_copy.cuh"

namespace spect {

constexpr int kConvThreads = 512;
constexpr int kConvWarps = kConvThreads / 32;
static_assert(kConvWarps <= kConvWarpsMax, "x-transform scratch sized for kConvWarpsMax warps");

struct ConvGeom {
  int nx, ny, nz;
  int Npx, Npz, logNpx, logNpz;
  int padup, padleft;
  int hx, hz;        // PSF half widths (px-1)/2, (pz-1)/2: extent of the folds
  int Q, QS;         // stored z-columns (max(1, Npz/2)) and B row stride (Q+1)
  int CX, logCX;     // lanes per x transform
  int CZ, logCZ;     // lanes per z transform
};

struct Conv2Args {
  ConvGeom g;
  const float* P;       // forward input planes  [nv][ny][nz][nx]
  float* T;             // adjoint output planes [nv][ny][nz][nx]
  const float* Hs;      // [nset][ny][Q+1][Npx]
  const int* vidx;      // [nv] plan view of each slot
  const int* viewset;   // [nview] spectrum set of each view
  const float2* Vs;     // adjoint input  [nv][Q][Npx] scrambled view spectra
  float2* VsOut;        // k_vspec2 output
  const float* views;   // k_vspec2 input [nv][nz][nx]
  int nv, chunkY, nchunks;
  float* part;          // forward output [nv][nchunks][nz][nx]
  float2* gB;           // per-CTA B slabs (nx*QS) when B is not in shared memory
  float2* gacc;         // per-CTA spectra slabs (Q*Npx) when they are not in registers
  const float2* tw;     // twiddles exp(-2 pi i m / SPECT_TW_N)
  int bsmem;
  const float* att;     // attenuation cache [view][y][z][x]; att_mul: applied on plane load (forward)
  int att_mul;
  int* err;             // set to 1 when a bounded wait gives up
  int vsplit;           // k_vspec2: column blocks per view (work items nv * vsplit)
};

struct Lanes {
  int l, g, gbase;  // lane in group, group in warp, first lane of group
};
__device__ __forceinline__ Lanes lanes_of(int lane, int logC) {
  Lanes L;
  L.l = lane & ((1 << logC) - 1);
  L.g = lane >> logC;
  L.gbase = L.g << logC;
  return L;
}

// Per-lane tables of the inverse z transform of a row pair (one entry per
// register k1 and lane, [k1 * 32 + lane]):
//   zgc  gather of the Hermitian spectrum from the stored columns: column c
//        and multipliers (mx, my, sy): a = (mx a.x + my a.y, sy a.y) turns the
//        stored value into the input of fft_inv (sy = -1: conjugate partner;
//        (1,0,0) / (0,1,0): the real DC / Nyquist packed in column 0)
//   zst  output sample z of register r: (z, or -1 outside the image; flags
//        1: z in the low fold range, 2: high fold range, 4: z == 0,
//        8: z == nz - 1)
//   xfl  per lane, bit r of: x of register r of the inverse x transform in
//        the low fold range, the high fold range, x == 0, x == nx - 1
struct ZTabs {
  const float4* zgc;
  const int2* zst;
  const int4* xfl;
};

template <int RZ>
__host__ __device__ constexpr int ztabs_bytes() {
  return RZ * 32 * 16 + RZ * 32 * 8 + 32 * 16;
}
template <int RX, int RZ>
__host__ __device__ constexpr int conv_tables_bytes() {
  return fft_tables_bytes(RX, RZ) + ztabs_bytes<RZ>();
}
__host__ __device__ constexpr int conv_tables_bytes_rt(int RX, int RZ) {
  return fft_tables_bytes(RX, RZ) + RZ * 32 * 16 + RZ * 32 * 8 + 32 * 16;
}

template <int RX, int RZ>
__device__ __forceinline__ ZTabs build_ztabs(const ConvGeom& g, void* at) {
  float4* zgc = reinterpret_cast<float4*>(at);
  int2* zst = reinterpret_cast<int2*>(zgc + RZ * 32);
  int4* xfl = reinterpret_cast<int4*>(zst + RZ * 32);
  for (int l = threadIdx.x; l < 32; l += blockDim.x) {
    const int CX = (RX > 1) ? 32 : g.CX, lx = l & (CX - 1);
    int lo = 0, hi = 0, first = 0, last = 0;
    for (int r = 0; r < RX; ++r) {
      const int x = lx + CX * r - g.padup;
      lo |= (x < 0 && x >= -g.hx) << r;
      hi |= (x >= g.nx && x < g.nx + g.hx) << r;
      first |= (x == 0) << r;
      last |= (x == g.nx - 1) << r;
    }
    xfl[l] = make_int4(lo, hi, first, last);
  }
  const int CZ = g.CZ, half = CZ >> 1;
  for (int e = threadIdx.x; e < RZ * 32; e += blockDim.x) {
    const int k1 = e >> 5, lz = (e & 31) & (CZ - 1);
    int c;
    float mx = 1.f, my = 0.f, sy = 1.f;
    if (CZ == 1) {
      c = 0;
      sy = 0.f;
    } else if ((lz & 1) == 0) {
      c = k1 * half + (lz >> 1);
      if (c == 0) sy = 0.f;
    } else if (k1 == 0 && lz == 1) {
      c = 0;
      mx = 0.f;
      my = 1.f;
      sy = 0.f;
    } else {
      int lp, rp;
      if (k1 > 0) {
        lp = lz ^ (CZ - 1);
        rp = RZ - k1;
      } else {
        lp = brev_rt((CZ - brev_rt(lz, g.logCZ)) & (CZ - 1), g.logCZ);
        rp = 0;
      }
      c = rp * half + (lp >> 1);
      sy = -1.f;
    }
    zgc[e] = make_float4(mx, my, sy, __int_as_float(c));
    const int z = lz + CZ * k1 - g.padleft;
    const int fl = ((z < 0 && z >= -g.hz) ? 1 : 0) | ((z >= g.nz && z < g.nz + g.hz) ? 2 : 0) | (z == 0 ? 4 : 0) |
                   (z == g.nz - 1 ? 8 : 0);
    zst[e] = make_int2((unsigned)z < (unsigned)g.nz ? z : -1, fl);
  }
  return ZTabs{zgc, zst, xfl};
}

// the z tables of a kernel with register counts RX, RZ (compile-time offset
// from the dynamic shared memory base: no pointer registers)
template <int RX, int RZ>
__device__ __forceinline__ ZTabs ztabs_of() {
  extern __shared__ float4 smem4[];
  const float4* zgc = reinterpret_cast<const float4*>(reinterpret_cast<const char*>(smem4) + fft_tables_bytes(RX, RZ));
  const int2* zst = reinterpret_cast<const int2*>(zgc + RZ * 32);
  return ZTabs{zgc, zst, reinterpret_cast<const int4*>(zst + RZ * 32)};
}

// shared memory: [FFT tables][z tables][B when bsmem]
// ZT: build the z tables (kernels with a folding inverse z transform)
template <int RX, int RZ, bool ZT = false>
__device__ __forceinline__ float2* conv_setup(const Conv2Args& a, FftTables* T) {
  extern __shared__ float4 smem4[];
  float2* base = reinterpret_cast<float2*>(smem4);
  *T = build_fft_tables(base, a.tw, RX, a.g.logNpx, RZ, a.g.logNpz);
  if (ZT) build_ztabs<RX, RZ>(a.g, reinterpret_cast<char*>(smem4) + fft_tables_bytes(RX, RZ));
  __syncthreads();
  if (a.bsmem) return base + conv_tables_bytes<RX, RZ>() / 8;
  return a.gB + (size_t)blockIdx.x * a.g.nx * a.g.QS;
}

// (x, z) walk of a thread over an nz x nx plane in steps of blockDim.x
struct PlaneWalk {
  int x0, z0, dx, dz;
  __device__ __forceinline__ PlaneWalk(int nx) {
    z0 = threadIdx.x / nx;
    x0 = threadIdx.x - z0 * nx;
    dz = blockDim.x / nx;
    dx = blockDim.x - dz * nx;
  }
};

// visits the elements (k = z * nx + x) of an nz x nx plane that belong to
// this thread; when nx divides blockDim.x each thread keeps one column x
template <class F>
__device__ __forceinline__ void plane_walk(const ConvGeom& g, const PlaneWalk& W, F f) {
  const int nx = g.nx;
  if (W.dx == 0) {
    const int x = W.x0;
#pragma unroll 2
    for (int z = W.z0; z < g.nz; z += W.dz) f(z * nx + x, x, z);
  } else {
    const int n = g.nx * g.nz;
    int x = W.x0, z = W.z0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      f(k, x, z);
      x += W.dx;
      z += W.dz;
      if (x >= nx) {
        x -= nx;
        ++z;
      }
    }
  }
}

// real nz x nx plane (x fastest) -> real rows of B, times the attenuation
// plane `att` when given
__device__ __forceinline__ void load_plane(const ConvGeom& g, const PlaneWalk& W, float2* B,
                                           const float* __restrict__ src, const float* __restrict__ att) {
  float* Bf = reinterpret_cast<float*>(B);
  const int rs = 2 * g.QS;
  plane_walk(g, W, [&](int k, int x, int z) {
    Bf[x * rs + z] = att ? __fmul_rn(__ldg(src + k), __ldg(att + k)) : __ldg(src + k);
  });
}

// real rows of B -> nz x nx plane (x fastest) in global memory, times the
// attenuation plane staged in shared memory
__device__ __forceinline__ void store_plane_satt(const ConvGeom& g, const PlaneWalk& W, const float2* B,
                                                 float* __restrict__ dst, const float* satt) {
  const float* Bf = reinterpret_cast<const float*>(B);
  const int rs = 2 * g.QS;
  plane_walk(g, W, [&](int k, int x, int z) { dst[k] = __fmul_rn(satt[k], Bf[x * rs + z]); });
}

// real rows of B -> nz x nx plane (x fastest) in global memory, times the
// attenuation plane `att` when given
__device__ __forceinline__ void store_plane(const ConvGeom& g, const PlaneWalk& W, const float2* B,
                                            float* __restrict__ dst, const float* __restrict__ att) {
  const float* Bf = reinterpret_cast<const float*>(B);
  const int rs = 2 * g.QS;
  plane_walk(g, W, [&](int k, int x, int z) {
    dst[k] = att ? __fmul_rn(__ldg(att + k), Bf[x * rs + z]) : Bf[x * rs + z];
  });
}

// Per-lane index tables, computed once per kernel.
//   zrd[r]  z source of register r for the forward z transform (clamped, or
//           -1 outside the image when zero padding)
//   zg[k1]  stored-column gather code for the inverse z transform:
//           (c << 2) | mode, mode 0 b[c], 1 conj(b[c]), 2 real b[c].x, 3 real b[c].y
//   xrd[r]  B row offset (x * QS) read by register r of the x transform
//           (clamped, or -1 outside the image when zero padding)
//   xwr[r]  B row offset written by register r after the inverse x transform
//           (-1 when cropped away)
template <int RX, int RZ>
struct LaneTables {
  int zrd[RZ], zg[RZ], xrd[RX], xwr[RX];
  // READ: zrd, xrd (forward transforms); WRITE: zg, xwr (inverse transforms)
  __device__ __forceinline__ void init(const ConvGeom& g, int lane, bool zeropad, bool read = true,
                                       bool write = true) {
    const int lz = lane & (g.CZ - 1), lx = lane & (g.CX - 1);
    const int CZ = g.CZ, half = CZ >> 1;
    if (read) {
#pragma unroll
      for (int r = 0; r < RZ; ++r) {
        int zc = lz + CZ * r - g.padleft;
        if (zeropad) zrd[r] = ((unsigned)zc < (unsigned)g.nz) ? zc : -1;
        else zrd[r] = min(max(zc, 0), g.nz - 1);
      }
#pragma unroll
      for (int r = 0; r < RX; ++r) {
        int x = lx + g.CX * r - g.padup;
        if (zeropad) xrd[r] = ((unsigned)x < (unsigned)g.nx) ? x * g.QS : -1;
        else xrd[r] = min(max(x, 0), g.nx - 1) * g.QS;
      }
    }
    if (!write) return;
#pragma unroll
    for (int k1 = 0; k1 < RZ; ++k1) {
      int code;
      if (CZ == 1) {
        code = 2;
      } else if ((lz & 1) == 0) {
        const int c = k1 * half + (lz >> 1);
        code = (c == 0) ? 2 : (c << 2);
      } else if (k1 == 0 && lz == 1) {
        code = 3;
      } else {
        int lp, rp;
        if (k1 > 0) {
          lp = lz ^ (CZ - 1);
          rp = RZ - k1;
        } else {
          lp = brev_rt((CZ - brev_rt(lz, g.logCZ)) & (CZ - 1), g.logCZ);
          rp = 0;
        }
        code = ((rp * half + (lp >> 1)) << 2) | 1;
      }
      zg[k1] = code;
    }
#pragma unroll
    for (int r = 0; r < RX; ++r) {
      int x = lx + g.CX * r - g.padup;
      xwr[r] = ((unsigned)x < (unsigned)g.nx) ? x * g.QS : -1;
    }
  }
};

// z transform of row pairs (x0, x0+1), in place in B: real rows -> stored
// columns.  ZEROPAD: zero padding (adjoint) instead of replication.
// psrc0: source lane of register 0's spectrum partner (z_partner_lane).
// Every lane stores its two unpacked values to a column: even lanes to
// k1 * half + lane/2, odd lanes (whose values duplicate an even lane's
// conjugates) to the unused column Q; lane 0 packs the Nyquist value of lane 1
// beside the DC value in column 0.
__device__ __forceinline__ int z_partner_lane(const ConvGeom& g, const Lanes& L) {
  return L.gbase + brev_rt((g.CZ - brev_rt(L.l, g.logCZ)) & (g.CZ - 1), g.logCZ);
}

template <int RZ, bool ZEROPAD>
__device__ __forceinline__ void zfft_rows_fwd(const ConvGeom& g, float2* B, const FftTables& TT, int warp,
                                              int lane, const int (&zrd)[RZ], int psrc0) {
  const Lanes L = lanes_of(lane, g.logCZ);
  const int CZ = RZ > 1 ? 32 : g.CZ, GZ = 32 >> g.logCZ, units = kConvWarps * GZ;
  const int npairs = g.nx >> 1, iters = (npairs + units - 1) / units;
  float* Bf = reinterpret_cast<float*>(B);
  const int rs = 2 * g.QS, QS = g.QS, half = CZ >> 1;
  const bool odd = (L.l & 1) != 0;
  const int cbase = odd ? g.Q : (L.l >> 1);
  for (int it = 0; it < iters; ++it) {
    const int rp = it * units + warp * GZ + L.g;
    const bool active = rp < npairs;
    const int x0 = 2 * min(rp, npairs - 1);
    const float* r0 = Bf + x0 * rs;
    const float* r1 = r0 + rs;
    float2 v[RZ];
#pragma unroll
    for (int r = 0; r < RZ; ++r) {
      const int zc = zrd[r];
      if (ZEROPAD) v[r] = (zc >= 0) ? make_float2(r0[zc], r1[zc]) : make_float2(0.f, 0.f);
      else v[r] = make_float2(r0[zc], r1[zc]);
    }
    __syncwarp();
    fft_fwd<RZ>(v, L.l, g.logCZ, TT, TT.rz + L.l);
    // partners: register k1 <-> RZ-k1 in lane l ^ (CZ-1); register 0 via psrc0
    float2 p[RZ];
    p[0] = shfl2(v[0], psrc0);
#pragma unroll
    for (int k1 = 1; k1 < RZ; ++k1) p[k1] = shfl_xor2(v[RZ - k1], CZ - 1);
    float2 A[RZ], Bb[RZ];
#pragma unroll
    for (int k1 = 0; k1 < RZ; ++k1) {
      // two real rows from one complex transform
      A[k1] = make_float2(0.5f * (v[k1].x + p[k1].x), 0.5f * (v[k1].y - p[k1].y));
      Bb[k1] = make_float2(0.5f * (v[k1].y + p[k1].y), 0.5f * (p[k1].x - v[k1].x));
    }
    float2* b0 = B + x0 * QS;
    float2* b1 = b0 + QS;
    if (CZ == 1) {
      if (active) {
        b0[0] = make_float2(A[0].x, 0.f);
        b1[0] = make_float2(Bb[0].x, 0.f);
      }
    } else {
      const float nyA = __shfl_sync(0xffffffffu, A[0].x, L.gbase + 1);
      const float nyB = __shfl_sync(0xffffffffu, Bb[0].x, L.gbase + 1);
      if (L.l == 0) {
        A[0].y = nyA;
        Bb[0].y = nyB;
      }
      if (active) {
#pragma unroll
        for (int k1 = 0; k1 < RZ; ++k1) {
          const int c = odd ? cbase : cbase + k1 * half;
          b0[c] = A[k1];
          b1[c] = Bb[k1];
        }
      }
    }
    __syncwarp();
  }
}

// Hermitian z-spectrum of the row pair from the stored columns, in the
// scrambled input order of fft_inv: v = Z0 + i Z1 (ZTabs::zgc + lane)
template <int RZ>
__device__ __forceinline__ void gather_zspec(const float2* b0, const float2* b1, const float4* zgc,
                                             float2 (&v)[RZ]) {
#pragma unroll
  for (int k1 = 0; k1 < RZ; ++k1) {
    const float4 t = zgc[k1 * 32];
    const int c = __float_as_int(t.w);
    const float2 a = b0[c], b = b1[c];
    const float ax = fmaf(t.x, a.x, t.y * a.y), ay = t.z * a.y;
    const float bx = fmaf(t.x, b.x, t.y * b.y), by = t.z * b.y;
    v[k1] = make_float2(ax - by, ay + bx);
  }
}

// Hermitian z-spectrum of the row pair from the stored columns, in the
// scrambled input order of fft_inv: v = Z0 + i Z1 (gather codes: LaneTables::zg;
// the forward kernels' chunk-end inverse, where registers are scarcer)
template <int RZ>
__device__ __forceinline__ void gather_zspec_codes(const float2* b0, const float2* b1, const int (&zg)[RZ],
                                             float2 (&v)[RZ]) {
#pragma unroll
  for (int k1 = 0; k1 < RZ; ++k1) {
    const int code = zg[k1], c = code >> 2, mode = code & 3;
    float2 a = b0[c], b = b1[c];
    if (mode == 1) {
      a.y = -a.y;
      b.y = -b.y;
    } else if (mode >= 2) {
      const bool hiq = mode == 3;
      a = make_float2(hiq ? a.y : a.x, 0.f);
      b = make_float2(hiq ? b.y : b.x, 0.f);
    }
    v[k1] = make_float2(a.x - b.y, a.y + b.x);
  }
}

template <int R>
__device__ __forceinline__ float2 group_sum(float2 s, int logC_rt) {
  const int logC = (R > 1) ? 5 : logC_rt;
#pragma unroll
  for (int q = 0; q < 5; ++q)
    if (q < logC) s = cadd(s, shfl_xor2(s, 1 << q));
  return s;
}

// inverse z transform of row pairs: stored columns -> real rows (in place).
// FOLD: adjoint of the replicate padding: the padded samples are summed into
// the edge samples.  Of the padded samples only the hz next to the image can
// be non-zero (zero-padded input, PSF half width hz, no wrap-around since the
// pads are >= hz), so only those are summed; the rest hold FFT round-off.
// gather and store through the shared-memory z tables (ZTabs)
template <int RZ, bool FOLD>
__device__ __forceinline__ void zfft_rows_inv(const ConvGeom& g, float2* B, const FftTables& TT, int warp,
                                              int lane, const ZTabs& Z) {
  const Lanes L = lanes_of(lane, g.logCZ);
  const int GZ = 32 >> g.logCZ, units = kConvWarps * GZ;
  const int npairs = g.nx >> 1, iters = (npairs + units - 1) / units;
  float* Bf = reinterpret_cast<float*>(B);
  const int rs = 2 * g.QS, QS = g.QS;
  for (int it = 0; it < iters; ++it) {
    const int rp = it * units + warp * GZ + L.g;
    const bool active = rp < npairs;
    const int x0 = 2 * min(rp, npairs - 1);
    float2 v[RZ];
    gather_zspec<RZ>(B + x0 * QS, B + (x0 + 1) * QS, Z.zgc + lane, v);
    __syncwarp();
    fft_inv<RZ>(v, L.l, g.logCZ, TT, TT.rz + L.l);
    float2 lo = make_float2(0.f, 0.f), hi = make_float2(0.f, 0.f);
    if (FOLD) {
#pragma unroll
      for (int r = 0; r < RZ; ++r) {
        const int fl = Z.zst[r * 32 + lane].y;
        if (fl & 1) lo = cadd(lo, v[r]);
        if (fl & 2) hi = cadd(hi, v[r]);
      }
      lo = group_sum<RZ>(lo, g.logCZ);
      hi = group_sum<RZ>(hi, g.logCZ);
    }
    if (active) {
      float* r0 = Bf + x0 * rs;
      float* r1 = r0 + rs;
#pragma unroll
      for (int r = 0; r < RZ; ++r) {
        const int2 e = Z.zst[r * 32 + lane];
        const int z = e.x;
        if (z >= 0) {
          float2 w = v[r];
          if (FOLD) {
            if (e.y & 4) w = cadd(w, lo);
            if (e.y & 8) w = cadd(w, hi);
          }
          r0[z] = w.x;
          r1[z] = w.y;
        }
      }
    }
    __syncwarp();
  }
}

// inverse z transform of row pairs: stored columns -> real rows (in place),
// gathering with the register codes zg (the forward kernels' chunk end).
// FOLD: adjoint of the replicate padding: the padded samples are summed into
// the edge samples.  Of the padded samples only the hz next to the image can
// be non-zero (zero-padded input, PSF half width hz, no wrap-around since the
// pads are >= hz), so only those are summed; the rest hold FFT round-off.
template <int RZ, bool FOLD>
__device__ __forceinline__ void zfft_rows_inv_codes(const ConvGeom& g, float2* B, const FftTables& TT, int warp,
                                              int lane, const int (&zg)[RZ]) {
  const Lanes L = lanes_of(lane, g.logCZ);
  const int CZ = g.CZ, GZ = 32 >> g.logCZ, units = kConvWarps * GZ;
  const int npairs = g.nx >> 1, iters = (npairs + units - 1) / units;
  float* Bf = reinterpret_cast<float*>(B);
  const int rs = 2 * g.QS, QS = g.QS;
  for (int it = 0; it < iters; ++it) {
    const int rp = it * units + warp * GZ + L.g;
    const bool active = rp < npairs;
    const int x0 = 2 * min(rp, npairs - 1);
    float2 v[RZ];
    gather_zspec_codes<RZ>(B + x0 * QS, B + (x0 + 1) * QS, zg, v);
    __syncwarp();
    fft_inv<RZ>(v, L.l, g.logCZ, TT, TT.rz + L.l);
    float2 lo = make_float2(0.f, 0.f), hi = make_float2(0.f, 0.f);
    if (FOLD) {
#pragma unroll
      for (int r = 0; r < RZ; ++r) {
        int z = L.l + CZ * r - g.padleft;
        if (z < 0 && z >= -g.hz) lo = cadd(lo, v[r]);
        else if (z >= g.nz && z < g.nz + g.hz) hi = cadd(hi, v[r]);
      }
      lo = group_sum<RZ>(lo, g.logCZ);
      hi = group_sum<RZ>(hi, g.logCZ);
    }
    if (active) {
      float* r0 = Bf + x0 * rs;
      float* r1 = r0 + rs;
#pragma unroll
      for (int r = 0; r < RZ; ++r) {
        int z = L.l + CZ * r - g.padleft;
        if ((unsigned)z < (unsigned)g.nz) {
          float2 w = v[r];
          if (FOLD) {
            if (z == 0) w = cadd(w, lo);
            if (z == g.nz - 1) w = cadd(w, hi);
          }
          r0[z] = w.x;
          r1[z] = w.y;
        }
      }
    }
    __syncwarp();
  }
}

// point-wise product with the plane's PSF spectrum (scrambled order).
// PACKED (warp-uniform): this warp holds column 0 in group 0.
template <int RX>
__device__ __forceinline__ void apply_psf(float2 (&v)[RX], const float* __restrict__ h, const float* __restrict__ hb,
                                          const Lanes& L, int logCX, bool packed_warp, bool col0) {
  const int CX = (RX > 1) ? 32 : (1 << logCX);
  if constexpr (RX == 8) {
    // 256-point layout (fftx256_fwd): the partner X[-k] is in the same lane
    if (packed_warp && col0) {
      float2 p[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) p[r] = v[7 - r];
      if (L.l == 0) {
        p[0] = v[0];
        p[1] = v[3];
        p[2] = v[2];
        p[3] = v[1];
#pragma unroll
        for (int r = 4; r < 8; ++r) p[r] = v[11 - r];
      }
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const float al = __ldg(h + r * 32), be = __ldg(hb + r * 32);
        v[r] = make_float2(al * v[r].x + be * p[r].x, al * v[r].y - be * p[r].y);
      }
      return;
    }
#pragma unroll
    for (int k1 = 0; k1 < RX; ++k1) v[k1] = cscale(v[k1], __ldg(h + k1 * CX));
    return;
  }
  if (packed_warp) {
    // Y' = alpha Y + beta conj(Y(-k)); registers k1 and RX-k1 are partners
    const int src0 = L.gbase + brev_rt((CX - brev_rt(L.l, logCX)) & (CX - 1), logCX);
    const float2 p0 = shfl2(v[0], src0);
    if (col0) v[0] = make_float2(__ldg(h) * v[0].x + __ldg(hb) * p0.x, __ldg(h) * v[0].y - __ldg(hb) * p0.y);
#pragma unroll
    for (int k1 = 1; k1 <= RX / 2; ++k1) {
      const int k2 = RX - k1;
      const float2 pa = shfl_xor2(v[k2], CX - 1);  // partner of register k1
      const float2 pb = shfl_xor2(v[k1], CX - 1);  // partner of register k2
      if (col0) {
        float al = __ldg(h + k1 * CX), be = __ldg(hb + k1 * CX);
        v[k1] = make_float2(al * v[k1].x + be * pa.x, al * v[k1].y - be * pa.y);
        if (k2 != k1) {
          al = __ldg(h + k2 * CX);
          be = __ldg(hb + k2 * CX);
          v[k2] = make_float2(al * v[k2].x + be * pb.x, al * v[k2].y - be * pb.y);
        }
      }
    }
    if (col0) return;
  }
#pragma unroll
  for (int k1 = 0; k1 < RX; ++k1) v[k1] = cscale(v[k1], __ldg(h + k1 * CX));
}

// ------------------------------------------------------------------------
// forward: persistent over items (slot, depth chunk)
template <int RX, int RZ, bool REGACC, bool STAGE>
__global__ void __launch_bounds__(kConvThreads, 1) k_conv_fwd2(Conv2Args a) {
  const ConvGeom& g = a.g;
  FftTables TT;
  float2* B = conv_setup<RX, RZ>(a, &TT);
  // STAGE: the next plane (and its attenuation) is bulk-copied into shared
  // staging buffers while the current one is transformed
  const int nplane = g.nz * g.nx;
  float* sP = reinterpret_cast<float*>(B + (size_t)g.nx * g.QS);
  float* sA = sP + nplane;
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(sA + (a.att_mul ? nplane : 0));
  unsigned phase = 0;
  auto issue = [&](int item, int y) {
    const int sl = item / a.nchunks;
    const float* src = a.P + ((size_t)sl * g.ny + y) * nplane;
    const float* asrc = a.att_mul ? a.att + ((size_t)a.vidx[sl] * g.ny + y) * nplane : nullptr;
    tma_planes(bar, sP, src, sA, asrc, (unsigned)(nplane * sizeof(float)));
  };
  if (STAGE) {
    if (threadIdx.x == 0) {
      mbar_init(bar);
      if ((int)blockIdx.x < a.nv * a.nchunks) issue(blockIdx.x, ((int)blockIdx.x % a.nchunks) * a.chunkY);
    }
    __syncthreads();
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2* const xw = TT.xscr ? TT.xscr + warp * kXScr : nullptr;  // x-transform scratch
  const Lanes L = lanes_of(lane, g.logCX);
  const int CX = (RX > 1) ? 32 : g.CX, GX = 32 / CX, units = kConvWarps * GX, Q = g.Q, Npx = g.Npx;
  const int JC = (Q + units - 1) / units;
  constexpr int JM = RZ > 1 ? RZ : 1;
  const int nitems = a.nv * a.nchunks;
  float2 acc[REGACC ? JM : 1][RX];
  float2* gacc = a.gacc + (size_t)blockIdx.x * Q * Npx;
  const PlaneWalk W(g.nx);
  LaneTables<RX, RZ> T;
  T.init(g, lane, false, true, false);
  const int zp0 = z_partner_lane(g, lanes_of(lane, g.logCZ));
  for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
    const int slot = item / a.nchunks, ch = item - slot * a.nchunks;
    const int y0 = ch * a.chunkY, y1 = min(g.ny, y0 + a.chunkY);
    const float* Pv = a.P + (size_t)slot * g.ny * g.nz * g.nx;
    const float* Hv = a.Hs + (size_t)a.viewset[a.vidx[slot]] * g.ny * (Q + 1) * Npx;
    for (int y = y0; y < y1; ++y) {
      if (STAGE) {
        // the block barrier also frees B from the previous plane
        if (__syncthreads_or(!mbar_wait(bar, phase))) {
          // a copy that never completed: flag it, give it one more bounded
          // wait, and leave the block
          if (threadIdx.x == 0) {
            atomicExch(a.err, 1);
            mbar_wait(bar, phase);
          }
          return;
        }
        phase ^= 1u;
        float* Bf = reinterpret_cast<float*>(B);
        const int rs = 2 * g.QS;
        if (a.att_mul)
          plane_walk(g, W, [&](int k, int x, int z) { Bf[x * rs + z] = __fmul_rn(sP[k], sA[k]); });
        else
          plane_walk(g, W, [&](int k, int x, int z) { Bf[x * rs + z] = sP[k]; });
        __syncthreads();
        if (threadIdx.x == 0) {  // prefetch the next plane of this CTA
          if (y + 1 < y1) issue(item, y + 1);
          else if (item + (int)gridDim.x < nitems)
            issue(item + gridDim.x, ((item + (int)gridDim.x) % a.nchunks) * a.chunkY);
        }
      } else {
        __syncthreads();
        load_plane(g, W, B, Pv + (size_t)y * g.nz * g.nx,
                   a.att_mul ? a.att + ((size_t)a.vidx[slot] * g.ny + y) * g.nz * g.nx : nullptr);
        __syncthreads();
      }
      zfft_rows_fwd<RZ, false>(g, B, TT, warp, lane, T.zrd, zp0);
      __syncthreads();
      const float* Hy = Hv + (size_t)y * (Q + 1) * Npx;
#pragma unroll
      for (int j = 0; j < JM; ++j) {
        if (j < JC) {
          const int c = j * units + warp * GX + L.g;
          const bool active = c < Q;
          const int cc = min(c, Q - 1);
          float2 v[RX];
#pragma unroll
          for (int r = 0; r < RX; ++r) v[r] = B[T.xrd[r] + cc];
          float hp[RX];  // PSF spectrum loads issued before the transform
#pragma unroll
          for (int k1 = 0; k1 < RX; ++k1) hp[k1] = __ldg(Hy + (size_t)cc * Npx + L.l + k1 * CX);
          fftx_fwd<RX>(v, L.l, g.logCX, TT, TT.rx + L.l, xw);
          if (j == 0 && warp == 0) {
            apply_psf<RX>(v, Hy + (size_t)cc * Npx + L.l, Hy + (size_t)Q * Npx + L.l, L, g.logCX, true, cc == 0);
          } else {
#pragma unroll
            for (int k1 = 0; k1 < RX; ++k1) v[k1] = cscale(v[k1], hp[k1]);
          }
          if (active) {
            if (REGACC) {
#pragma unroll
              for (int k1 = 0; k1 < RX; ++k1) acc[REGACC ? j : 0][k1] = (y == y0) ? v[k1] : cadd(acc[REGACC ? j : 0][k1], v[k1]);
            } else {
              float2* ga = gacc + (size_t)c * Npx + L.l;
#pragma unroll
              for (int k1 = 0; k1 < RX; ++k1) ga[k1 * CX] = (y == y0) ? v[k1] : cadd(ga[k1 * CX], v[k1]);
            }
          }
        }
      }
    }
    // chunk end: inverse x transform, crop to nx rows
    __syncthreads();
    LaneTables<RX, RZ> TW;
    TW.init(g, lane, false, false, true);
#pragma unroll
    for (int j = 0; j < JM; ++j) {
      if (j < JC) {
        const int c = j * units + warp * GX + L.g;
        const bool active = c < Q;
        float2 v[RX];
        if (REGACC) {
#pragma unroll
          for (int k1 = 0; k1 < RX; ++k1) v[k1] = acc[REGACC ? j : 0][k1];
        } else {
          const float2* ga = gacc + (size_t)min(c, Q - 1) * Npx + L.l;
#pragma unroll
          for (int k1 = 0; k1 < RX; ++k1) v[k1] = ga[k1 * CX];
        }
        fftx_inv<RX>(v, L.l, g.logCX, TT, TT.rx + L.l, xw);
        if (active) {
#pragma unroll
          for (int r = 0; r < RX; ++r)
            if (TW.xwr[r] >= 0) B[TW.xwr[r] + c] = v[r];
        }
      }
    }
    __syncthreads();
    zfft_rows_inv_codes<RZ, false>(g, B, TT, warp, lane, TW.zg);
    __syncthreads();
    store_plane(g, W, B, a.part + ((size_t)slot * a.nchunks + ch) * g.nz * g.nx, nullptr);
  }
}

// ------------------------------------------------------------------------
// scrambled spectrum of each zero-padded view: VsOut[slot][c][k1*CX + l]
template <int RX, int RZ>
__global__ void __launch_bounds__(kConvThreads, 1) k_vspec2(Conv2Args a) {
  const ConvGeom& g = a.g;
  FftTables TT;
  float2* B = conv_setup<RX, RZ>(a, &TT);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2* const xw = TT.xscr ? TT.xscr + warp * kXScr : nullptr;  // x-transform scratch
  const Lanes L = lanes_of(lane, g.logCX);
  const int CX = (RX > 1) ? 32 : g.CX, GX = 32 / CX, units = kConvWarps * GX, Q = g.Q, Npx = g.Npx;
  const PlaneWalk W(g.nx);
  LaneTables<RX, RZ> T;
  T.init(g, lane, true);
  const int zp0 = z_partner_lane(g, lanes_of(lane, g.logCZ));
  // work item = (slot, block of columns): the z transforms are repeated per
  // block so that a few views still spread over the whole GPU
  const int vs = max(1, a.vsplit), cpb = (Q + vs - 1) / vs;
  for (int item = blockIdx.x; item < a.nv * vs; item += gridDim.x) {
    const int slot = item / vs, cb0 = (item - slot * vs) * cpb, cb1 = min(Q, cb0 + cpb);
    __syncthreads();
    load_plane(g, W, B, a.views + (size_t)slot * g.nz * g.nx, nullptr);
    __syncthreads();
    zfft_rows_fwd<RZ, true>(g, B, TT, warp, lane, T.zrd, zp0);
    __syncthreads();
    for (int it = 0; it * units < cb1 - cb0; ++it) {
      const int c = cb0 + it * units + warp * GX + L.g;
      const int cc = min(c, cb1 - 1);
      float2 v[RX];
#pragma unroll
      for (int r = 0; r < RX; ++r) v[r] = (T.xrd[r] >= 0) ? B[T.xrd[r] + cc] : make_float2(0.f, 0.f);
      fftx_fwd<RX>(v, L.l, g.logCX, TT, TT.rx + L.l, xw);
      if (c < cb1) {
        float2* o = a.VsOut + ((size_t)slot * Q + c) * Npx + L.l;
#pragma unroll
        for (int k1 = 0; k1 < RX; ++k1) o[k1 * CX] = v[k1];
      }
    }
  }
}

// ------------------------------------------------------------------------
// adjoint: persistent over items (slot, depth chunk); T[slot][y][z][x]
template <int RX, int RZ, bool REGACC, bool STAGE>
__global__ void __launch_bounds__(kConvThreads, 1) k_conv_adj2(Conv2Args a) {
  const ConvGeom& g = a.g;
  FftTables TT;
  float2* B = conv_setup<RX, RZ, true>(a, &TT);
  // STAGE: the attenuation plane of each output plane is bulk-copied into
  // shared memory while the plane is transformed, and multiplied in on store.
  // Shared memory: [FFT tables][B when bsmem][attenuation plane][mbarrier]
  const int nplane = g.nz * g.nx;
  extern __shared__ float4 smem4[];
  float* sA = reinterpret_cast<float*>(reinterpret_cast<char*>(smem4) + conv_tables_bytes<RX, RZ>() +
                                       (a.bsmem ? sizeof(float2) * (size_t)g.nx * g.QS : 0));
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(sA + nplane);
  unsigned phase = 0;
  if (STAGE) {
    if (threadIdx.x == 0) mbar_init(bar);
    __syncthreads();
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2* const xw = TT.xscr ? TT.xscr + warp * kXScr : nullptr;  // x-transform scratch
  const Lanes L = lanes_of(lane, g.logCX);
  const int CX = (RX > 1) ? 32 : g.CX, GX = 32 / CX, units = kConvWarps * GX, Q = g.Q, Npx = g.Npx;
  const int JC = (Q + units - 1) / units;
  constexpr int JM = RZ > 1 ? RZ : 1;
  const int nitems = a.nv * a.nchunks;
  float2 vs[REGACC ? JM : 1][RX];
  const PlaneWalk W(g.nx);
  LaneTables<RX, RZ> T;
  T.init(g, lane, false);
  for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
    const int slot = item / a.nchunks, ch = item - slot * a.nchunks;
    const int y0 = ch * a.chunkY, y1 = min(g.ny, y0 + a.chunkY);
    const float* Hv = a.Hs + (size_t)a.viewset[a.vidx[slot]] * g.ny * (Q + 1) * Npx;
    const float2* Vsl = a.Vs + (size_t)slot * Q * Npx;
    if (REGACC) {
#pragma unroll
      for (int j = 0; j < JM; ++j) {
        if (j < JC) {
          const int cc = min(j * units + warp * GX + L.g, Q - 1);
#pragma unroll
          for (int k1 = 0; k1 < RX; ++k1) vs[REGACC ? j : 0][k1] = Vsl[(size_t)cc * Npx + L.l + k1 * CX];
        }
      }
    }
    for (int y = y0; y < y1; ++y) {
      const float* Hy = Hv + (size_t)y * (Q + 1) * Npx;
      __syncthreads();
      if (STAGE && threadIdx.x == 0) {
        fence_proxy_async();
        mbar_expect(bar, (unsigned)(nplane * sizeof(float)));
        bulk_copy(bar, sA, a.att + ((size_t)a.vidx[slot] * g.ny + y) * nplane, (unsigned)(nplane * sizeof(float)));
      }
#pragma unroll
      for (int j = 0; j < JM; ++j) {
        if (j < JC) {
          const int c = j * units + warp * GX + L.g;
          const bool active = c < Q;
          const int cc = min(c, Q - 1);
          float2 v[RX];
#pragma unroll
          for (int k1 = 0; k1 < RX; ++k1)
            v[k1] = REGACC ? vs[REGACC ? j : 0][k1] : Vsl[(size_t)cc * Npx + L.l + k1 * CX];
          apply_psf<RX>(v, Hy + (size_t)cc * Npx + L.l, Hy + (size_t)Q * Npx + L.l, L, g.logCX,
                        j == 0 && warp == 0, cc == 0);
          fftx_inv<RX>(v, L.l, g.logCX, TT, TT.rx + L.l, xw);
          // adjoint of the replicate padding along x (fold masks: ZTabs::xfl)
          const int4 xm = ztabs_of<RX, RZ>().xfl[lane];
          float2 lo = make_float2(0.f, 0.f), hi = make_float2(0.f, 0.f);
#pragma unroll
          for (int r = 0; r < RX; ++r) {
            if ((xm.x >> r) & 1) lo = cadd(lo, v[r]);
            if ((xm.y >> r) & 1) hi = cadd(hi, v[r]);
          }
          lo = group_sum<RX>(lo, g.logCX);
          hi = group_sum<RX>(hi, g.logCX);
          if (active) {
#pragma unroll
            for (int r = 0; r < RX; ++r) {
              const int off = T.xwr[r];
              if (off >= 0) {
                float2 w = v[r];
                if ((xm.z >> r) & 1) w = cadd(w, lo);
                if ((xm.w >> r) & 1) w = cadd(w, hi);
                B[off + c] = w;
              }
            }
          }
        }
      }
      __syncthreads();
      zfft_rows_inv<RZ, true>(g, B, TT, warp, lane, ztabs_of<RX, RZ>());
      if (STAGE) {
        if (__syncthreads_or(!mbar_wait(bar, phase))) {
          if (threadIdx.x == 0) {
            atomicExch(a.err, 1);
            mbar_wait(bar, phase);
          }
          return;
        }
        phase ^= 1u;
        store_plane_satt(g, W, B, a.T + ((size_t)slot * g.ny + y) * g.nz * g.nx, sA);
      } else {
        __syncthreads();
        store_plane(g, W, B, a.T + ((size_t)slot * g.ny + y) * g.nz * g.nx, nullptr);
      }
    }
  }
}

}  // namespace spect
