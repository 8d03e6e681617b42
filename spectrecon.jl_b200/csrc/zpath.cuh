// zpath.cuh -- the fused SPECT projector pair on z-fastest layouts (sm_100a),
// for the common case: :two rotation, cached attenuation, separable (rank-1)
// PSF planes.
//
// Layouts (float32, z fastest; nzp = nz rounded up to 16; every entry with
// z >= nz is zero):
//   IZ    [L][L][nzp]        image on the zero-padded rotation grid
//                            (L = nx + 2 pad, pad = ceil(1 + nx sqrt2/2 - nx/2),
//                            src/plan-rotate.jl:56): voxel (x, y, z) at
//                            ((y + pad) L + x + pad) nzp + z.  The ring is
//                            zero, so bilinear taps need no bounds tests.
//   ATT   [view][y][x][nzp]  attenuation exp(-dy (sum_{j<y} mu_j + mu_y/2)) on
//                            the view's rotated grid (src/project.jl:103-113)
//   T     [slot][y][x][nzp]  adjoint planes att .* conv_adj(view) of a group
//   views [slot][nz][nx]     the reference's views[nx, nz, nview], unchanged
//
// k_zfwd   project! (src/project.jl:77-135): work item (slot, depth chunk);
//          per plane y the block gathers the rotated image (imrotate! :two,
//          src/rotatez.jl:331-362) column by column from IZ, multiplies the
//          attenuation plane (bulk-copied one plane ahead) and writes the
//          z-pass buffer directly; then the z pass and the x pass of the
//          replicate-boundary convolution that fft_conv! computes
//          (src/fft_convolve.jl:33-55).  The x-pass outputs stay in
//          registers across the chunk (the depth sum, src/project.jl:127-130).
//          The rotated volume never leaves the SM.
// k_zadj   backproject! (src/backproject.jl:69-124), convolution half: per
//          plane the x pass and z pass of fft_conv_adj! (src/fft_convolve.jl:
//          82-130) of the view, times the attenuation, stored as T.
// k_zrot_adj  imrotate_adj! :two (src/rotatez.jl:390-416) and the view sum
//          (src/backproject.jl:146-153): output-stationary gather.  A group of
//          8 lanes owns one image column (x, y) over all z (8 lanes x ZPL) and
//          sums, over the group's views in order, the bilinear weights of the
//          rotated-grid points whose footprint covers it: the exact transpose
//          of the forward sampling, without atomics.  The EM update
//          (src/ml-os-em.jl:111-126) is its epilogue.
//
// Convolution passes.  fft_conv! equals the replicate-boundary convolution
// out[i] = sum_{m<p} w[m] in[clamp(i - h + m)] with the reversed factor w
// (the plan factors each PSF plane as a[d] b[e]).  Here the input line sits
// zero-padded in shared memory, data starting at an offset D0 = h rounded up
// to 4, and the weights are shifted right by D0 - h, so an 8-output task reads
// a window of 16-byte-aligned float4s; the clamped boundary is added as tail
// terms: the edge value times EL[i] = sum_{m < h - i} w[m] (i < h) or
// ER[n-1-i] = sum_{m > h + n-1-i} w[m] (i > n-1-h).  The adjoint passes are the
// zero-padded correlations with the factors themselves plus the folded padding
// at the two ends (cL_k, cR_k: sums of the factor beyond k), as the reference's
// padding adjoint does.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "bulk_copy.cuh"
#include "zpath_api.h"

namespace spect {

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }

// 8 taps of one 8-output task: o[k] += w[s] e[s + k], with the block's
// weights (w0, w1) and e = (p, q, r, t) the 16 consecutive window elements
// starting at the block's first tap
__device__ __forceinline__ void zfma8(float4 w0, float4 w1, float4 p, float4 q, float4 r, float4 t, float (&o)[8]) {
  const float ws[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
  const float e[16] = {p.x, p.y, p.z, p.w, q.x, q.y, q.z, q.w, r.x, r.y, r.z, r.w, t.x, t.y, t.z, t.w};
#pragma unroll
  for (int s = 0; s < 8; ++s)
#pragma unroll
    for (int k = 0; k < 8; ++k) o[k] = fmaf(ws[s], e[s + k], o[k]);
}

// one 8-output task over a zero-padded line, the window in nblk blocks of 8
// taps (nblk <= 9): o[k] += sum_{m < 8 nblk} w[m] line[k + m] (line and w
// 16-byte aligned; reads line[0, 8 nblk + 8)).  Fully unrolled with a uniform
// early exit: the window quads alternate between two register pairs by name
// (no loop counter or register moves), and the next block's weights are
// loaded one block ahead, so a block's FMAs never start by waiting for them
// (PF = false: loaded at the block, for callers short of registers).
template <bool PF = true>
__device__ __forceinline__ void zpassu(const float* __restrict__ w, int nblk, const float* line, float (&o)[8]) {
  float4 a = ld4(line), b = ld4(line + 4), c, d;
  float4 wa0 = ld4(w), wa1 = ld4(w + 4), wb0, wb1;
#pragma unroll
  for (int k = 0; k < 10; k += 2) {
    if (k >= nblk) break;
    c = ld4(line + 8 * k + 8);
    d = ld4(line + 8 * k + 12);
    if (PF && k + 1 < nblk) {
      wb0 = ld4(w + 8 * k + 8);
      wb1 = ld4(w + 8 * k + 12);
    }
    if (!PF && k > 0) {
      wa0 = ld4(w + 8 * k);
      wa1 = ld4(w + 8 * k + 4);
    }
    zfma8(wa0, wa1, a, b, c, d, o);
    if (k + 1 >= nblk) break;
    a = ld4(line + 8 * k + 16);
    b = ld4(line + 8 * k + 20);
    if (PF && k + 2 < nblk) {
      wa0 = ld4(w + 8 * k + 16);
      wa1 = ld4(w + 8 * k + 20);
    }
    if (!PF) {
      wb0 = ld4(w + 8 * k + 8);
      wb1 = ld4(w + 8 * k + 12);
    }
    zfma8(wb0, wb1, c, d, a, b, o);
  }
}

// q = t / n for 0 <= t < 2^20, 1 <= n <= 4096, with r = 1/n rounded to float:
// (t + 1/2) / n is at least 1/(2n) from an integer, far above the rounding
// error of (t + 1/2) * r, so truncation gives the exact quotient
__device__ __forceinline__ int zdiv(int t, float r) { return (int)(((float)t + 0.5f) * r); }

// ------------------------------------------------------------------------
// Layout changes between the caller's image [z][y][x] and IZ.
// k_to_iz: IZ interior (and its z padding) from img; grid (ceil(nx/32),
// ny, ceil(nzp/32)), block (32, 8).
__global__ void __launch_bounds__(256) k_to_iz(ZGeom g, const float* __restrict__ img, float* __restrict__ iz) {
  __shared__ float tile[32][33];
  const int x0 = blockIdx.x * 32, y = blockIdx.y, z0 = blockIdx.z * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int k = ty; k < 32; k += 8) {  // tile[z][x], coalesced over x
    const int z = z0 + k, x = x0 + tx;
    tile[k][tx] = (z < g.nz && x < g.nx) ? img[((size_t)z * g.ny + y) * g.nx + x] : 0.f;
  }
  __syncthreads();
  for (int k = ty; k < 32; k += 8) {  // IZ column x, coalesced over z
    const int x = x0 + k, z = z0 + tx;
    if (x < g.nx && z < g.nzp) iz[((size_t)(y + g.pad) * g.L + x + g.pad) * g.nzp + z] = tile[tx][k];
  }
}

// k_from_iz: dst (caller layout) from the IZ interior.  mode 0: dst = v;
// 1: dst = v, zeros -> +Inf (EM sensitivity, src/ml-os-em.jl:111-114);
// 2: dst = dst * (v / asum) (EM update, asum in the caller layout).
__global__ void __launch_bounds__(256) k_from_iz(ZGeom g, const float* __restrict__ iz, float* dst,
                                                 const float* __restrict__ asum, int mode) {
  __shared__ float tile[32][33];
  const int x0 = blockIdx.x * 32, y = blockIdx.y, z0 = blockIdx.z * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int k = ty; k < 32; k += 8) {  // tile[x][z], coalesced over z
    const int x = x0 + k, z = z0 + tx;
    tile[k][tx] = (x < g.nx && z < g.nz) ? iz[((size_t)(y + g.pad) * g.L + x + g.pad) * g.nzp + z] : 0.f;
  }
  __syncthreads();
  for (int k = ty; k < 32; k += 8) {  // caller row (z, y), coalesced over x
    const int z = z0 + k, x = x0 + tx;
    if (z < g.nz && x < g.nx) {
      const size_t o = ((size_t)z * g.ny + y) * g.nx + x;
      float v = tile[tx][k];
      if (mode == 1 && v == 0.f) v = __int_as_float(0x7f800000);
      if (mode == 2) v = dst[o] * (v / asum[o]);
      dst[o] = v;
    }
  }
}

// k_t_to_z: adjoint planes of the split kernels ([plane][nz][nx], plane =
// slot * ny + y) into the z-fastest T layout ([plane][nx][nzp], zeros for
// z >= nz) that k_zrot_adj reads, multiplied by the attenuation when the
// convolution has not applied it (att non-null, the same product as the
// reference's a_y .* conv_adj); grid (ceil(nx/32), planes, ceil(nzp/32)),
// block (32, 8).
__global__ void __launch_bounds__(256) k_t_to_z(ZGeom g, const float* __restrict__ src, float* __restrict__ dst,
                                                const float* __restrict__ att, const int* __restrict__ vidx) {
  __shared__ float tile[32][33];
  const int x0 = blockIdx.x * 32, pl = blockIdx.y, z0 = blockIdx.z * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const float* s = src + (size_t)pl * g.nz * g.nx;
  float* d = dst + (size_t)pl * g.nx * g.nzp;
  // att (split layout [view][y][z][x]) given: the planes are not premultiplied yet
  const float* av = att ? att + ((size_t)vidx[pl / g.ny] * g.ny + pl % g.ny) * g.nz * g.nx : nullptr;
  for (int k = ty; k < 32; k += 8) {  // tile[z][x], coalesced over x
    const int z = z0 + k, x = x0 + tx;
    const size_t o = (size_t)z * g.nx + x;
    tile[k][tx] = (z < g.nz && x < g.nx) ? (av ? __fmul_rn(av[o], s[o]) : s[o]) : 0.f;
  }
  __syncthreads();
  for (int k = ty; k < 32; k += 8) {  // column x, coalesced over z
    const int x = x0 + k, z = z0 + tx;
    if (x < g.nx && z < g.nzp) d[(size_t)x * g.nzp + z] = tile[tx][k];
  }
}

// ------------------------------------------------------------------------
// Geometry of rotated-grid point (x, y) of a view, with the forward
// sampling's products and sums in the same order and rounding
// (RotPos::pos): the IZ offset of its lower-left tap and the four bilinear
// weights (w00, w10, w01, w11); theta == 0 copies (the reference's forward
// shortcut).  Every sample of the cropped grid lies inside the padded grid;
// a point outside it (impossible for finite angles) contributes nothing.
__device__ __forceinline__ void zgeo(const ZGeom& g, float cs, float sn, bool ident, int x, int y, float4& w,
                                     int& off) {
  int j1 = x, j2 = y;
  w = make_float4(1.f, 0.f, 0.f, 0.f);
  if (!ident) {
    const float di = __fsub_rn((float)x, g.c0), dj = __fsub_rn((float)y, g.c0);
    const float s1 = __fadd_rn(g.c0, __fsub_rn(__fmul_rn(cs, di), __fmul_rn(sn, dj)));
    const float s2 = __fadd_rn(g.c0, __fadd_rn(__fmul_rn(sn, di), __fmul_rn(cs, dj)));
    const float f1 = floorf(s1), f2 = floorf(s2);
    const float t1 = __fsub_rn(s1, f1), t2 = __fsub_rn(s2, f2);
    const float u1 = __fsub_rn(1.0f, t1), u2 = __fsub_rn(1.0f, t2);
    j1 = (int)f1;
    j2 = (int)f2;
    w = make_float4(__fmul_rn(u1, u2), __fmul_rn(t1, u2), __fmul_rn(u1, t2), __fmul_rn(t1, t2));
    if (j1 < -g.pad || j1 > g.nx + g.pad - 2 || j2 < -g.pad || j2 > g.nx + g.pad - 2) {
      j1 = j2 = 0;
      w = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
  off = ((j2 + g.pad) * g.L + j1 + g.pad) * g.nzp;
}

// Attenuation cache in the ATT layout: block (column x, view v), one thread
// per z (nzp threads); each walks y and scans the rotated mu-map (bilinear
// sample of the IZ-laid-out mu-map with bilinear()'s fmul/fadd order), as
// k_atten_build does.
__global__ void __launch_bounds__(256) k_zatten(ZGeom g, const float* __restrict__ muz,
                                               const float4* __restrict__ rot, float dy, float* __restrict__ att) {
  const int x = blockIdx.x, v = blockIdx.y, z = threadIdx.x;
  if (z >= g.nzp) return;
  const float4 r = rot[v];
  const bool ident = r.z != 0.f;
  const float mdy = -dy;
  float prefix = 0.f;
  const size_t Lz = (size_t)g.L * g.nzp;
  for (int y = 0; y < g.ny; ++y) {
    float4 w;
    int off;
    zgeo(g, r.x, r.y, ident, x, y, w, off);
    const float* p = muz + off + z;
    float m = __fmul_rn(w.x, p[0]);
    m = __fadd_rn(m, __fmul_rn(w.y, p[g.nzp]));
    m = __fadd_rn(m, __fmul_rn(w.z, p[Lz]));
    m = __fadd_rn(m, __fmul_rn(w.w, p[Lz + g.nzp]));
    const float e = __fadd_rn(prefix, __fmul_rn(0.5f, m));
    att[(((size_t)v * g.ny + y) * g.nx + x) * g.nzp + z] = z < g.nz ? expf(__fmul_rn(e, mdy)) : 0.f;
    prefix = __fadd_rn(prefix, m);
  }
}

// ------------------------------------------------------------------------
// k_zfwd<NT, NTH>: persistent forward, one block per SM, NTH threads; NT
// x-pass tasks per thread, all of a plane's x tasks resident
// (NT * NTH >= nz * nx / 8) since their outputs accumulate over the chunk.
// Per plane: wait for the staged attenuation plane and weights, sample
// geometry of the plane's nx rotated-grid columns, gather into ZB, z pass
// into XB, x pass into registers (three block barriers per plane).
template <int NT, int NTH>
__global__ void __launch_bounds__(NTH, 1) k_zfwd(ZArgs a) {
  extern __shared__ float4 smem4[];
  const ZGeom& g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz, nzp = g.nzp, hs = g.hs, ts = g.ts;
  float* const base = reinterpret_cast<float*>(smem4);
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(base);
  float* const sA = base + 4;                   // attenuation plane [x][nzp]
  float* const sW = sA + (size_t)nx * nzp;      // weights then tails (staging)
  float* const Hw0 = sW + hs + ts;              // working weights, two planes
  float2* const PA = reinterpret_cast<float2*>(Hw0 + 2 * (hs + ts));
  float2* const PB = PA + nx;
  float4* const geoW = reinterpret_cast<float4*>(PB + ny);
  int* const geoO = reinterpret_cast<int*>(geoW + nx);
  float* const ZB = reinterpret_cast<float*>(geoO + zround(nx, 4));  // [x][ast], data rows R0..R0+nz-1
  float* const XB = ZB + (size_t)nx * g.ast;                          // [z][bs], data columns C0..C0+nx-1
  const int tid = threadIdx.x;
  const int nitems = a.nv * a.nchunks;
  const unsigned abytes = (unsigned)((size_t)nx * nzp * sizeof(float));
  auto issue = [&](int item, int y) {  // one thread: attenuation plane, weights, tails of plane y
    const int sl = item / a.nchunks, v = a.vidx[sl], set = a.viewset[v];
    fence_proxy_async();
    mbar_expect(bar, abytes + (unsigned)((hs + ts) * sizeof(float)));
    bulk_copy(bar, sA, a.att + ((size_t)v * ny + y) * nx * nzp, abytes);
    bulk_copy(bar, sW, a.H + ((size_t)set * ny + y) * (2 * hs), (unsigned)(hs * sizeof(float)));
    bulk_copy(bar, sW + hs, a.E + ((size_t)set * ny + y) * (2 * ts), (unsigned)(ts * sizeof(float)));
  };
  // the padded buffers start zero; only their data rows / columns are written later
  for (size_t k = tid; k < (size_t)nx * g.ast + (size_t)nz * g.bs; k += NTH) ZB[k] = 0.f;
  if (tid == 0) {
    mbar_init(bar);
    if ((int)blockIdx.x < nitems) issue(blockIdx.x, ((int)blockIdx.x % a.nchunks) * a.chunkY);
  }
  __syncthreads();
  const int nzb = (nz + 7) / 8, ztasks = nx * nzb, nz4 = (nz + 3) / 4, units = nx * nz4;
  const int xtasks = nz * (nx / 8);
  const size_t Lz = (size_t)g.L * nzp;
  const int ast = g.ast, bs = g.bs, R0 = g.R0, C0 = g.C0, hz = g.hz, hx = g.hx;
  const int zblk = g.zpw / 8, xblk = g.xpw / 8, zpw = g.zpw;
  const float rnx = 1.0f / nx, rnz = 1.0f / nz, rnz4 = 1.0f / nz4;
  unsigned phase = 0;
  int yb = 0;  // working-weight buffer of the current plane
  float acc[NT][8];
  for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
    const int slot = item / a.nchunks, ch = item - slot * a.nchunks;
    const int v = a.vidx[slot];
    const int y0 = ch * a.chunkY, y1 = min(ny, y0 + a.chunkY);
    const float4 r = a.rot[v];
    const float cs = r.x, sn = r.y;
    const bool ident = r.z != 0.f;
    // position tables of this view, the products of RotPos::pos (the
    // previous item's geometry was done before its last barrier)
    for (int e = tid; e < nx + ny; e += NTH) {
      const int o = e < nx ? e : e - nx;
      const float d = __fsub_rn((float)o, g.c0);
      if (e < nx) PA[o] = make_float2(__fmul_rn(cs, d), __fmul_rn(sn, d));
      else PB[o] = make_float2(__fmul_rn(sn, d), __fmul_rn(cs, d));
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < NT; ++i)
#pragma unroll
      for (int k = 0; k < 8; ++k) acc[i][k] = 0.f;
    for (int y = y0; y < y1; ++y) {
      const bool ok = mbar_wait(bar, phase);
      phase ^= 1u;
      float* const Hw = Hw0 + yb * (hs + ts);
      // sample geometry of plane y, one rotated-grid column per thread
      if (tid < nx) {
        int j1 = tid, j2 = y;
        float4 w = make_float4(1.f, 0.f, 0.f, 0.f);
        if (!ident) {
          const float2 pa = PA[tid], pb = PB[y];
          const float s1 = __fadd_rn(g.c0, __fsub_rn(pa.x, pb.x)), s2 = __fadd_rn(g.c0, __fadd_rn(pa.y, pb.y));
          const float f1 = floorf(s1), f2 = floorf(s2);
          const float t1 = __fsub_rn(s1, f1), t2 = __fsub_rn(s2, f2);
          const float u1 = __fsub_rn(1.0f, t1), u2 = __fsub_rn(1.0f, t2);
          j1 = (int)f1;
          j2 = (int)f2;
          w = make_float4(__fmul_rn(u1, u2), __fmul_rn(t1, u2), __fmul_rn(u1, t2), __fmul_rn(t1, t2));
          if (j1 < -g.pad || j1 > nx + g.pad - 2 || j2 < -g.pad || j2 > nx + g.pad - 2) {
            j1 = j2 = 0;
            w = make_float4(0.f, 0.f, 0.f, 0.f);
          }
        }
        geoW[tid] = w;
        geoO[tid] = ((j2 + g.pad) * g.L + j1 + g.pad) * nzp;
      }
      for (int k = tid; k < hs + ts; k += NTH) Hw[k] = sW[k];
      if (__syncthreads_or(!ok)) {
        if (tid == 0) {
          atomicExch(a.err, 1);
          mbar_wait(bar, phase ^ 1u);
        }
        return;
      }
      // rotated, attenuated plane into ZB (column x, rows R0 + z), four z at a time
      for (int u = tid; u < units; u += NTH) {
        const int x = zdiv(u, rnz4), zg = u - x * nz4;
        const float4 w = geoW[x];
        const float* p = a.img + geoO[x] + 4 * zg;
        const float4 t0 = ld4(p), t1 = ld4(p + nzp), t2 = ld4(p + Lz), t3 = ld4(p + Lz + nzp);
        const float4 at = ld4(sA + x * nzp + 4 * zg);
        float4 o;
        o.x = __fmul_rn(fmaf(w.w, t3.x, fmaf(w.z, t2.x, fmaf(w.y, t1.x, __fmul_rn(w.x, t0.x)))), at.x);
        o.y = __fmul_rn(fmaf(w.w, t3.y, fmaf(w.z, t2.y, fmaf(w.y, t1.y, __fmul_rn(w.x, t0.y)))), at.y);
        o.z = __fmul_rn(fmaf(w.w, t3.z, fmaf(w.z, t2.z, fmaf(w.y, t1.z, __fmul_rn(w.x, t0.z)))), at.z);
        o.w = __fmul_rn(fmaf(w.w, t3.w, fmaf(w.z, t2.w, fmaf(w.y, t1.w, __fmul_rn(w.x, t0.w)))), at.w);
        st4(ZB + x * ast + R0 + 4 * zg, o);
      }
      __syncthreads();
      if (tid == 0) {  // next plane of this block into the staging buffers
        if (y + 1 < y1) issue(item, y + 1);
        else if (item + (int)gridDim.x < nitems) issue(item + gridDim.x, ((item + (int)gridDim.x) % a.nchunks) * a.chunkY);
      }
      // z pass: task (x, z block) -> XB rows z, column C0 + x
      const float* ELz = Hw + hs;
      const float* ERz = ELz + hz;
      for (int t = tid; t < ztasks; t += NTH) {
        const int zb = zdiv(t, rnx), x = t - zb * nx, z0 = 8 * zb;
        float o[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) o[k] = 0.f;
        const float* col = ZB + x * ast;
        zpassu<(NT <= 2)>(Hw, zblk, col + z0, o);
        if (z0 < hz) {  // clamped rows above the plane
          const float e0 = col[R0];
#pragma unroll
          for (int k = 0; k < 8; ++k)
            if (z0 + k < hz) o[k] = fmaf(ELz[z0 + k], e0, o[k]);
        }
        if (z0 + 8 > nz - hz) {  // clamped rows below
          const float e1 = col[R0 + nz - 1];
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            const int kk = nz - 1 - z0 - k;
            if (kk >= 0 && kk < hz) o[k] = fmaf(ERz[kk], e1, o[k]);
          }
        }
        float* xo = XB + z0 * bs + C0 + x;
#pragma unroll
        for (int k = 0; k < 8; ++k)
          if (z0 + k < nz) xo[k * bs] = o[k];
      }
      __syncthreads();
      // x pass, accumulated over the chunk
      const float* ELx = ERz + hz;
      const float* ERx = ELx + hx;
#pragma unroll
      for (int i = 0; i < NT; ++i) {
        const int t = tid + i * NTH;
        if (t < xtasks) {
          const int xb = zdiv(t, rnz), z = t - xb * nz, x0 = 8 * xb;
          const float* row = XB + z * bs;
          zpassu<(NT <= 2)>(Hw + zpw, xblk, row + x0, acc[i]);
          if (x0 < hx) {
            const float e0 = row[C0];
#pragma unroll
            for (int k = 0; k < 8; ++k)
              if (x0 + k < hx) acc[i][k] = fmaf(ELx[x0 + k], e0, acc[i][k]);
          }
          if (x0 + 8 > nx - hx) {
            const float e1 = row[C0 + nx - 1];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
              const int kk = nx - 1 - x0 - k;
              if (kk < hx) acc[i][k] = fmaf(ERx[kk], e1, acc[i][k]);
            }
          }
        }
      }
      yb ^= 1;
    }
    // partial view of this chunk: part[slot][ch][z][x]
    float* out = a.part + ((size_t)slot * a.nchunks + ch) * nz * nx;
#pragma unroll
    for (int i = 0; i < NT; ++i) {
      const int t = tid + i * NTH;
      if (t < xtasks) {
        const int xb = zdiv(t, rnz), z = t - xb * nz;
        float* o = out + (size_t)z * nx + 8 * xb;
        st4(o, make_float4(acc[i][0], acc[i][1], acc[i][2], acc[i][3]));
        st4(o + 4, make_float4(acc[i][4], acc[i][5], acc[i][6], acc[i][7]));
      }
    }
  }
}

// ------------------------------------------------------------------------
// k_zadj<NT, NTH>: adjoint convolution; work items (slot, depth chunk); the
// view is loaded zero-padded once per item; per plane the adjoint weights and
// folds are bulk-copied two planes deep; x pass (view rows) -> WB, z pass (WB
// columns) -> times the attenuation column (16-byte global loads issued at
// the task's start) -> T.  NT only sets how the x tasks are interleaved.
template <int NT, int NTH>
__global__ void __launch_bounds__(NTH, 1) k_zadj(ZArgs a) {
  extern __shared__ float4 smem4[];
  const ZGeom& g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz, nzp = g.nzp, hs = g.hs, ts = g.ts;
  float* const base = reinterpret_cast<float*>(smem4);
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(base);  // two barriers
  const int sts = hs + ts;                 // one stage: weights, folds
  float* const stage = base + 4;
  float* const VB = stage + 2 * sts;
  float* const WB = VB + (size_t)nz * g.bs;
  const int tid = threadIdx.x;
  const int nitems = a.nv * a.nchunks;
  auto issue = [&](int item, int y, int b) {  // one thread
    const int sl = item / a.nchunks, v = a.vidx[sl], set = a.viewset[v];
    float* st = stage + b * sts;
    fence_proxy_async();
    mbar_expect(&bar[b], (unsigned)((hs + ts) * sizeof(float)));
    bulk_copy(&bar[b], st, a.H + ((size_t)set * ny + y) * (2 * hs) + hs, (unsigned)(hs * sizeof(float)));
    bulk_copy(&bar[b], st + hs, a.E + ((size_t)set * ny + y) * (2 * ts) + ts, (unsigned)(ts * sizeof(float)));
  };
  auto next = [&](int& item, int& y) {
    const int yend = min(ny, (item % a.nchunks) * a.chunkY + a.chunkY);
    if (y + 1 < yend) {
      ++y;
    } else {
      item += gridDim.x;
      y = (item % a.nchunks) * a.chunkY;
    }
  };
  // WB rows outside the data rows stay zero
  for (int x = tid / 32; x < nx; x += NTH / 32)
    for (int r = tid & 31; r < g.ast; r += 32)
      if (r < g.R0 || r >= g.R0 + nz) WB[(size_t)x * g.ast + r] = 0.f;
  int qi = blockIdx.x, qy = (blockIdx.x % a.nchunks) * a.chunkY;  // plane P0
  int i1 = qi, y1q = qy;
  next(i1, y1q);  // P1
  if (tid == 0) {
    mbar_init(&bar[0]);
    mbar_init(&bar[1]);
    if (qi < nitems) {
      issue(qi, qy, 0);
      if (i1 < nitems) issue(i1, y1q, 1);
    }
  }
  __syncthreads();
  qi = i1;
  qy = y1q;
  next(qi, qy);  // P2: the next plane to issue
  if (!((int)blockIdx.x < nitems)) return;
  const int nzb = (nz + 7) / 8, ztasks = nx * nzb, xtasks = nz * (nx / 8);
  const int ast = g.ast, bs = g.bs, R0 = g.R0, C0 = g.C0, hz = g.hz, hx = g.hx;
  const int zblk = g.zpw / 8, xblk = g.xpw / 8;
  const float rnx = 1.0f / nx, rnz = 1.0f / nz;
  unsigned phases = 0u;
  int b = 0;
  for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
    const int slot = item / a.nchunks, ch = item - slot * a.nchunks;
    const int v = a.vidx[slot];
    const int y0 = ch * a.chunkY, y1 = min(ny, y0 + a.chunkY);
    // the view, zero-padded (the previous item's passes ended at a barrier)
    const float* V = a.views + (size_t)slot * nz * nx;
    for (int z = tid / 32; z < nz; z += NTH / 32) {
      float* row = VB + (size_t)z * g.bs;
      for (int c = tid & 31; c < g.bs; c += 32) row[c] = (c >= g.C0 && c < g.C0 + nx) ? V[z * nx + c - g.C0] : 0.f;
    }
    for (int y = y0; y < y1; ++y) {
      const unsigned par = (phases >> b) & 1u;
      if (__syncthreads_or(!mbar_wait(&bar[b], par))) {
        if (tid == 0) {
          atomicExch(a.err, 1);
          mbar_wait(&bar[b], par);
        }
        return;
      }
      phases ^= 1u << b;
      const float* st = stage + b * sts;
      const float* az = st;             // adjoint z weights (shifted)
      const float* ax = st + g.zpw;     // adjoint x weights (shifted)
      const float* cLx = st + hs;       // folds
      const float* cRx = cLx + g.hx;
      const float* cLz = cRx + g.hx;
      const float* cRz = cLz + g.hz;
      // x pass: task (z, x block) -> WB column x, row R0 + z
#pragma unroll
      for (int i = 0; i < NT; ++i)
        for (int t = tid + i * NTH; t < xtasks; t += NT * NTH) {
          const int xb = zdiv(t, rnz), z = t - xb * nz, x0 = 8 * xb;
          const float* row = VB + z * bs;
          float o[8];
#pragma unroll
          for (int k = 0; k < 8; ++k) o[k] = 0.f;
          zpassu(ax, xblk, row + x0, o);
          if (x0 == 0)
            for (int k = 0; k < hx; ++k) o[0] = fmaf(cLx[k], row[C0 + k], o[0]);
          if (x0 + 8 == nx)
            for (int k = 0; k < hx; ++k) o[7] = fmaf(cRx[k], row[C0 + nx - 1 - k], o[7]);
          float* w = WB + x0 * ast + R0 + z;
#pragma unroll
          for (int k = 0; k < 8; ++k) w[k * ast] = o[k];
        }
      __syncthreads();
      // z pass: task (x, z block) -> T column (x, y) of the slot
      const float* attv = a.att + (((size_t)v * ny + y) * nx) * nzp;
      float* Tp = a.T + (((size_t)slot * ny + y) * nx) * nzp;
      for (int t = tid; t < ztasks; t += NTH) {
        const int zb = zdiv(t, rnx), x = t - zb * nx, z0 = 8 * zb;
        const float4 a0 = ld4(attv + x * nzp + z0), a1 = ld4(attv + x * nzp + z0 + 4);
        const float* col = WB + x * ast;
        float o[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) o[k] = 0.f;
        zpassu(az, zblk, col + z0, o);
        if (z0 == 0)
          for (int k = 0; k < hz; ++k) o[0] = fmaf(cLz[k], col[R0 + k], o[0]);
        if (z0 <= nz - 1 && nz - 1 < z0 + 8) {
          const int kz = nz - 1 - z0;
          float s = 0.f;
          for (int k = 0; k < hz; ++k) s = fmaf(cRz[k], col[R0 + nz - 1 - k], s);
#pragma unroll
          for (int k = 0; k < 8; ++k)
            if (k == kz) o[k] += s;
        }
        float* dst = Tp + x * nzp + z0;
        st4(dst, make_float4(__fmul_rn(a0.x, o[0]), __fmul_rn(a0.y, o[1]), __fmul_rn(a0.z, o[2]),
                             __fmul_rn(a0.w, o[3])));
        st4(dst + 4, make_float4(__fmul_rn(a1.x, o[4]), __fmul_rn(a1.y, o[5]), __fmul_rn(a1.z, o[6]),
                                 __fmul_rn(a1.w, o[7])));
      }
      __syncthreads();
      if (tid == 0 && qi < nitems) issue(qi, qy, b);  // this stage is free again
      next(qi, qy);
      b ^= 1;
    }
  }
}

// ------------------------------------------------------------------------
// k_zrot_adj<ZPL>: two 8-lane groups of a warp own image column p = (j1, j2)
// (grid-stride), lane l of a group the z values l + 8 q, q < ZPL (nzp =
// 8 ZPL): one 32-byte sector per group and load, the candidate geometry shared
// by the group's 8 lanes.  The first group sums the even slots, the second
// the odd ones; a shuffle adds the two partial sums (a fixed order).  For
// every slot, the rotated-grid points (x, y) whose bilinear footprint contains
// (j1, j2) -- those with floor(s1) in {j1-1, j1} and floor(s2) in {j2-1, j2}
// -- lie within |cos| + |sin| of the inverse-rotated pixel centre, so the
// candidates are at most 3 x 3 points; each is tested with the forward's own
// position arithmetic and weighted with the forward's weight product.
// Epilogue (IZ layout): v = acc (+ prev); mode 1: zeros -> +Inf; mode 2:
// v = x * (v / asum); out = v (z < nz only; out may be prev or x).
template <int ZPL>
__global__ void __launch_bounds__(256) k_zrot_adj(ZGeom g, const float* __restrict__ T,
                                                 const float4* __restrict__ rot, const int* __restrict__ vidx, int nv,
                                                 const float* prev, float* out, const float* x,
                                                 const float* __restrict__ asum, int mode) {
  const int lane = threadIdx.x & 7, half = (threadIdx.x >> 3) & 1;
  const int npix = (gridDim.x * blockDim.x) >> 4;
  const int nx = g.nx, ny = g.ny, nzp = g.nzp;
  const float c0 = g.c0;
  // every warp runs the same number of iterations (the shuffle needs all lanes)
  for (int p0 = (blockIdx.x * blockDim.x + (threadIdx.x & ~31)) >> 4; p0 < nx * nx; p0 += npix) {
    const int p = min(p0 + ((threadIdx.x >> 4) & 1), nx * nx - 1);
    const bool own = p0 + ((threadIdx.x >> 4) & 1) < nx * nx;
    const int j2 = p / nx, j1 = p - j2 * nx;
    const float fj1 = (float)j1, fj2 = (float)j2;
    float acc[ZPL];
#pragma unroll
    for (int q = 0; q < ZPL; ++q) acc[q] = 0.f;
    for (int s = half; s < nv; s += 2) {
      const float4 r = rot[vidx[s]];
      const float cs = r.x, sn = r.y;
      const float d1 = fj1 - c0, d2 = fj2 - c0;
      const float xc = c0 + cs * d1 + sn * d2, yc = c0 - sn * d1 + cs * d2;
      const float rr = fabsf(cs) + fabsf(sn) + 0.01f;
      const int xlo = max(0, (int)ceilf(xc - rr)), xhi = min(nx - 1, (int)floorf(xc + rr));
      const int ylo = max(0, (int)ceilf(yc - rr)), yhi = min(ny - 1, (int)floorf(yc + rr));
      const float* Ts = T + (size_t)s * ny * nx * nzp + lane;
      // the candidates first (weights, column offsets; 0 for the invalid
      // ones), then their loads, so that a group has all of them in flight
      float cw[9];
      int co[9];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const int xx = min(xlo + i, nx - 1);
        const float di = __fsub_rn((float)xx, c0);
        const float ca = __fmul_rn(cs, di), cc = __fmul_rn(sn, di);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const int yy = min(ylo + k, ny - 1);
          const float dj = __fsub_rn((float)yy, c0);
          const float s1 = __fadd_rn(c0, __fsub_rn(ca, __fmul_rn(sn, dj)));
          const float s2 = __fadd_rn(c0, __fadd_rn(cc, __fmul_rn(cs, dj)));
          const bool ok = xlo + i <= xhi && ylo + k <= yhi && s1 >= fj1 - 1.f && s1 < fj1 + 1.f &&
                          s2 >= fj2 - 1.f && s2 < fj2 + 1.f;
          const float f1 = floorf(s1), f2 = floorf(s2);
          const float t1 = __fsub_rn(s1, f1), t2 = __fsub_rn(s2, f2);
          const float a1 = f1 == fj1 ? __fsub_rn(1.0f, t1) : t1;
          const float a2 = f2 == fj2 ? __fsub_rn(1.0f, t2) : t2;
          cw[3 * i + k] = ok ? __fmul_rn(a1, a2) : 0.f;
          co[3 * i + k] = ok ? (yy * nx + xx) * nzp : -1;
        }
      }
#pragma unroll
      for (int c = 0; c < 9; ++c)
        if (co[c] >= 0) {
          const float* tp = Ts + co[c];
#pragma unroll
          for (int q = 0; q < ZPL; ++q) acc[q] = fmaf(cw[c], tp[8 * q], acc[q]);
        }
    }
#pragma unroll
    for (int q = 0; q < ZPL; ++q) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], 8);  // even + odd slots
    if (half || !own) continue;
    const size_t o = ((size_t)(j2 + g.pad) * g.L + j1 + g.pad) * nzp + lane;
#pragma unroll
    for (int q = 0; q < ZPL; ++q) {
      if (lane + 8 * q < g.nz) {
        float v = acc[q];
        if (prev) v += prev[o + 8 * q];
        if (mode == 1 && v == 0.f) v = __int_as_float(0x7f800000);
        if (mode == 2) v = x[o + 8 * q] * (v / asum[o + 8 * q]);
        out[o + 8 * q] = v;
      }
    }
  }
}

}  // namespace spect
