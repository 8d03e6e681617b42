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
// The kernels for planes too large for these kernels' shared memory are in
// zstrip.cuh (same layouts and passes, over plane tiles).
// k_zrot_adj  imrotate_adj! :two (src/rotatez.jl:390-416) and the view sum
//          (src/backproject.jl:146-153): output-stationary gather.  Groups of
//          8 lanes own one image column (x, y) over all z (8 lanes x ZPL) and
//          sum, over their views in order, the bilinear weights of the
//          rotated-grid points whose footprint covers it: the exact transpose
//          of the forward sampling, without atomics.  The EM update
//          (src/ml-os-em.jl:111-126) is its epilogue.
//
// Convolution passes.  fft_conv! equals the replicate-boundary convolution
// out[i] = sum_{m<p} w[m] in[clamp(i - h + m)] with the reversed factor w
// (the plan factors each PSF plane as a[d] b[e]).  Here the input line sits
// zero-padded in shared memory, data starting at an offset D0 = h rounded up
// to 4, and the weights are shifted right by D0 - h, so a task of W = 8 or 16
// consecutive outputs reads a window of 16-byte-aligned float4s; the clamped
// boundary is added as tail terms: the edge value times EL[i] =
// sum_{m < h - i} w[m] (i < h) or ER[n-1-i] = sum_{m > h + n-1-i} w[m]
// (i > n-1-h).  The adjoint passes are the zero-padded correlations with the
// factors themselves plus the folded padding at the two ends (cL_k, cR_k:
// sums of the factor beyond k), as the reference's padding adjoint does.
// The plan zeroes the outer taps of each factor whose summed magnitude per
// side is within 2^-27 of the factor's (below Float32 resolution; a narrow
// Gaussian plane keeps a few of its p taps) and every table, tails and folds
// included, comes from those factors; per plane and pass a range table gives
// the 8-tap blocks that hold the kept taps, and only those are run.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "bulk_copy.cuh"
#include "zpath_api.h"

#ifndef ZFWD_GU
#define ZFWD_GU 2
#endif

namespace spect {

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
// 8-byte read-only global load issued only where pred holds; (0, 0) elsewhere
// (no memory access for those lanes).  p must be 8-byte aligned.
__device__ __forceinline__ float2 ldg2_if(const float* p, bool pred) {
  unsigned a, b;
  asm("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %3, 0;\n\tmov.b32 %0, 0;\n\tmov.b32 %1, 0;\n\t"
      "@q ld.global.nc.v2.b32 {%0, %1}, [%2];\n\t}"
      : "=r"(a), "=r"(b)
      : "l"(p), "r"((int)pred));
  return make_float2(__uint_as_float(a), __uint_as_float(b));
}

// one W-output task (W = 8 or 16) over a zero-padded line, the taps
// m in [4 b4, 4 b4 + 8 nblk) in blocks of 8 (nblk <= 9): o[k] += sum_m w[m]
// line[k + m] (line and w 16-byte aligned; reads line[4 b4, 4 b4 + 8 nblk +
// W)).  Fully unrolled with a uniform early exit; the window elements are
// named by constant indices (registers, no moves): per block two new quads
// of the line and two weight quads feed 8 W FMAs.  Every output sums its
// taps in ascending m, so W does not change the result.
template <int W>
__device__ __forceinline__ void zpassw(const float* __restrict__ w, int b4, int nblk, const float* line,
                                       float (&o)[W]) {
  w += 4 * b4;
  line += 4 * b4;
  float e[W + 8 * 9];
#pragma unroll
  for (int i = 0; i < W / 4; ++i) {
    const float4 q = ld4(line + 4 * i);
    e[4 * i] = q.x;
    e[4 * i + 1] = q.y;
    e[4 * i + 2] = q.z;
    e[4 * i + 3] = q.w;
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    if (k >= nblk) break;
    const float4 q0 = ld4(line + 8 * k + W), q1 = ld4(line + 8 * k + W + 4);
    e[8 * k + W] = q0.x;
    e[8 * k + W + 1] = q0.y;
    e[8 * k + W + 2] = q0.z;
    e[8 * k + W + 3] = q0.w;
    e[8 * k + W + 4] = q1.x;
    e[8 * k + W + 5] = q1.y;
    e[8 * k + W + 6] = q1.z;
    e[8 * k + W + 7] = q1.w;
    const float4 w0 = ld4(w + 8 * k), w1 = ld4(w + 8 * k + 4);
    const float ws[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
#pragma unroll
    for (int s2 = 0; s2 < 8; ++s2)
#pragma unroll
      for (int j = 0; j < W; ++j) o[j] = fmaf(ws[s2], e[8 * k + s2 + j], o[j]);
  }
}

// sum_{k < n} c[k] v[step k]: four partial sums over k mod 4, added as
// (s0 + s1) + (s2 + s3); four taps' loads per round are independent, so a
// round waits for one load latency
__device__ __forceinline__ float zfold(const float* c, const float* v, int step, int n) {
  float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
  int k = 0;
  for (; k + 4 <= n; k += 4) {
    s0 = fmaf(c[k], v[step * k], s0);
    s1 = fmaf(c[k + 1], v[step * (k + 1)], s1);
    s2 = fmaf(c[k + 2], v[step * (k + 2)], s2);
    s3 = fmaf(c[k + 3], v[step * (k + 3)], s3);
  }
  if (k < n) s0 = fmaf(c[k], v[step * k], s0);
  if (k + 1 < n) s1 = fmaf(c[k + 1], v[step * (k + 1)], s1);
  if (k + 2 < n) s2 = fmaf(c[k + 2], v[step * (k + 2)], s2);
  return (s0 + s1) + (s2 + s3);
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
// k_zfwd<NT, NTH, W>: persistent forward, one block per SM, NTH threads; NT
// x-pass tasks of W outputs per thread, all of a plane's x tasks resident
// (NT * NTH >= nz * nx / W) since their outputs accumulate over the chunk.
// The block walks its planes in sequence; the attenuation plane and weights
// of the next nsf planes are bulk-copied while plane p is worked on (stage
// q % nsf holds plane q).  Two block barriers per plane: phase A runs the z
// pass of plane p (ZB -> XB) and the sample geometry of plane p + 1; phase B
// the x pass of plane p (XB -> registers) and the gather of plane p + 1
// (rotated, attenuated image -> ZB).
template <int NT, int NTH, int W>
__global__ void __launch_bounds__(NTH, 1) k_zfwd(ZArgs a) {
  constexpr int GU = ZFWD_GU;  // gather units per thread and round (4 measured ~1 % faster, with spills in some shapes)
  extern __shared__ float4 smem4[];
  const ZGeom& g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz, nzp = g.nzp, hs = g.hs, ts = g.ts, nsf = g.nsf;
  float* const base = reinterpret_cast<float*>(smem4);
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(base);  // nsf barriers
  const int hts = hs + ts + 4;         // weights, tails, tap ranges of one plane (4 ints)
  const int sts = nx * nzp + hts;      // stage: attenuation plane [x][nzp], then those
  float* const stage = base + 4;
  float* const Hw0 = stage + nsf * sts;           // working weights, tails, ranges: two planes
  float4* const geoW = reinterpret_cast<float4*>(Hw0 + 2 * hts);
  int* const geoO = reinterpret_cast<int*>(geoW + nx);
  float* const ZB = reinterpret_cast<float*>(geoO + zround(nx, 4));  // [x][ast], data rows R0..R0+nz-1
  float* const XB = ZB + (size_t)nx * g.ast;                          // [z][bs], data columns C0..C0+nx-1
  const int tid = threadIdx.x;
  const int nitems = a.nv * a.nchunks;
  const float rnc = 1.0f / a.nchunks;
  auto slot_of = [&](int item) { return zdiv(item, rnc); };             // item / nchunks (items < 2^20)
  auto chunk_of = [&](int item) { return item - zdiv(item, rnc) * a.nchunks; };
  const unsigned abytes = (unsigned)((size_t)nx * nzp * sizeof(float));
  auto issue = [&](int item, int y, int s) {  // one thread: attenuation plane, weights, tails of plane y
    const int sl = slot_of(item), v = a.vidx[sl], set = a.viewset[v];
    float* sA = stage + s * sts;
    float* sW = sA + nx * nzp;
    fence_proxy_async();
    mbar_expect(&bar[s], abytes + (unsigned)(hts * sizeof(float)));
    bulk_copy(&bar[s], sA, a.att + ((size_t)v * ny + y) * nx * nzp, abytes);
    bulk_copy(&bar[s], sW, a.H + ((size_t)set * ny + y) * (2 * hs), (unsigned)(hs * sizeof(float)));
    bulk_copy(&bar[s], sW + hs, a.E + ((size_t)set * ny + y) * (2 * ts), (unsigned)(ts * sizeof(float)));
    bulk_copy(&bar[s], sW + hs + ts, a.R + ((size_t)set * ny + y) * 8, 4u * sizeof(int));
  };
  auto next = [&](int& item, int& y) {
    const int yend = min(ny, chunk_of(item) * a.chunkY + a.chunkY);
    if (y + 1 < yend) {
      ++y;
    } else {
      item += gridDim.x;
      y = chunk_of(item) * a.chunkY;
    }
  };
  // the padded buffers start zero; only their data rows / columns are written later
  for (size_t k = tid; k < (size_t)nx * g.ast + (size_t)nz * g.bs; k += NTH) ZB[k] = 0.f;
  int i0 = blockIdx.x, y0 = (blockIdx.x % a.nchunks) * a.chunkY;  // plane p
  int i1 = i0, y1 = y0;
  next(i1, y1);  // p + 1
  int iq = i1, yq = y1;  // the next plane to issue
  unsigned pend = 0u;    // stages with a copy issued and not yet waited for (same in every thread)
  if (tid == 0) {
    for (int s = 0; s < nsf; ++s) mbar_init(&bar[s]);
    if (i0 < nitems) issue(i0, y0, 0);
  }
  pend = 1u;
  if (nsf > 1) {
    if (tid == 0 && iq < nitems) issue(iq, yq, 1);
    if (iq < nitems) pend |= 2u;
    next(iq, yq);
  }
  __syncthreads();
  if (!(i0 < nitems)) return;
  const int nzb = (nz + W - 1) / W, ztasks = nx * nzb, nz4 = (nz + 3) / 4, units = nx * nz4;
  const int xtasks = nz * (nx / W);
  const size_t Lz = (size_t)g.L * nzp;
  const int ast = g.ast, bs = g.bs, R0 = g.R0, C0 = g.C0, hz = g.hz, hx = g.hx;
  const int zpw = g.zpw;
  const float rnx = 1.0f / nx, rnz = 1.0f / nz, rnz4 = 1.0f / nz4;
  unsigned phases = 0u;  // parity of each barrier's next wait
  // wait for stage s; false (every thread) when a wait gave up, after the
  // copies in flight have landed
  auto staged = [&](int s) {
    const bool ok = mbar_wait(&bar[s], (phases >> s) & 1u);
    if (ok) {
      phases ^= 1u << s;
      pend &= ~(1u << s);
    }
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(a.err, 1);
        for (int k = 0; k < nsf; ++k)
          if ((pend >> k) & 1u) mbar_wait(&bar[k], (phases >> k) & 1u);
      }
      return false;
    }
    return true;
  };
  // sample geometry of plane (item, y), one rotated-grid column per thread:
  // the position arithmetic of RotPos::pos with the view's (cos, sin)
  auto geometry = [&](int item, int y) {
    if (tid < nx) {
      const float4 r = a.rot[a.vidx[slot_of(item)]];
      int j1 = tid, j2 = y;
      float4 w = make_float4(1.f, 0.f, 0.f, 0.f);
      if (r.z == 0.f) {
        const float cs = r.x, sn = r.y;
        const float d1 = __fsub_rn((float)tid, g.c0), d2 = __fsub_rn((float)y, g.c0);
        const float s1 = __fadd_rn(g.c0, __fsub_rn(__fmul_rn(cs, d1), __fmul_rn(sn, d2)));
        const float s2 = __fadd_rn(g.c0, __fadd_rn(__fmul_rn(sn, d1), __fmul_rn(cs, d2)));
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
  };
  // staged weights of stage s into working buffer hb; rotated, attenuated
  // plane into ZB (column x, rows R0 + z), four z at a time
  auto gather = [&](int s, int hb) {
    const float* const sA = stage + s * sts;
    const float* const sW = sA + nx * nzp;
    float* const Hw = Hw0 + hb * hts;
    for (int k = tid; k < hs + ts; k += NTH) Hw[k] = sW[k];
    if (tid < 4) reinterpret_cast<int*>(Hw + hs + ts)[tid] = reinterpret_cast<const int*>(sW + hs + ts)[tid];
    // GU units per round, all their image loads issued before any is used
    for (int u0 = tid; u0 < units; u0 += GU * NTH) {
      float4 t[GU][4];
      int xs[GU], zs[GU];
#pragma unroll
      for (int j = 0; j < GU; ++j) {
        const int u = min(u0 + j * NTH, units - 1);  // a repeated last unit stores the same values
        xs[j] = zdiv(u, rnz4);
        zs[j] = u - xs[j] * nz4;
        const float* p = a.img + geoO[xs[j]] + 4 * zs[j];
        t[j][0] = ld4(p);
        t[j][1] = ld4(p + nzp);
        t[j][2] = ld4(p + Lz);
        t[j][3] = ld4(p + Lz + nzp);
      }
#pragma unroll
      for (int j = 0; j < GU; ++j) {
        const float4 w = geoW[xs[j]];
        const float4 at = ld4(sA + xs[j] * nzp + 4 * zs[j]);
        const float4 t0 = t[j][0], t1 = t[j][1], t2 = t[j][2], t3 = t[j][3];
        float4 o;
        o.x = __fmul_rn(fmaf(w.w, t3.x, fmaf(w.z, t2.x, fmaf(w.y, t1.x, __fmul_rn(w.x, t0.x)))), at.x);
        o.y = __fmul_rn(fmaf(w.w, t3.y, fmaf(w.z, t2.y, fmaf(w.y, t1.y, __fmul_rn(w.x, t0.y)))), at.y);
        o.z = __fmul_rn(fmaf(w.w, t3.z, fmaf(w.z, t2.z, fmaf(w.y, t1.z, __fmul_rn(w.x, t0.z)))), at.z);
        o.w = __fmul_rn(fmaf(w.w, t3.w, fmaf(w.z, t2.w, fmaf(w.y, t1.w, __fmul_rn(w.x, t0.w)))), at.w);
        st4(ZB + xs[j] * ast + R0 + 4 * zs[j], o);
      }
    }
  };
  float acc[NT][W];
#pragma unroll
  for (int i = 0; i < NT; ++i)
#pragma unroll
    for (int k = 0; k < W; ++k) acc[i][k] = 0.f;
  // the stage that plane p's copy used is free again: the plane nsf ahead
  auto refill = [&](int s) {
    if (iq < nitems) {
      if (tid == 0) issue(iq, yq, s);
      pend |= 1u << s;
    }
    next(iq, yq);
  };
  // prologue: plane p's geometry and staged data, its gather
  geometry(i0, y0);
  if (!staged(0)) return;
  gather(0, 0);
  __syncthreads();
  refill(0);
  int hb = 0, s1 = nsf > 1 ? 1 : 0;  // working-weight buffer of plane p, stage of plane p + 1
  for (;;) {
    const bool h1 = i1 < nitems;
    const float* Hw = Hw0 + hb * hts;
    const int4 rg = *reinterpret_cast<const int4*>(Hw + hs + ts);  // tap ranges: z pass, x pass
    // phase A: z pass of p, task (x, z block) -> XB rows z, column C0 + x
    const float* ELz = Hw + hs;
    const float* ERz = ELz + hz;
    for (int t = tid; t < ztasks; t += NTH) {
      const int zb = zdiv(t, rnx), x = t - zb * nx, z0 = W * zb;
      float o[W];
#pragma unroll
      for (int k = 0; k < W; ++k) o[k] = 0.f;
      const float* col = ZB + x * ast;
      zpassw<W>(Hw, rg.x, rg.y, col + z0, o);
      if (z0 < hz) {  // clamped rows above the plane
        const float e0 = col[R0];
#pragma unroll
        for (int k = 0; k < W; ++k)
          if (z0 + k < hz) o[k] = fmaf(ELz[z0 + k], e0, o[k]);
      }
      if (z0 + W > nz - hz) {  // clamped rows below
        const float e1 = col[R0 + nz - 1];
#pragma unroll
        for (int k = 0; k < W; ++k) {
          const int kk = nz - 1 - z0 - k;
          if (kk >= 0 && kk < hz) o[k] = fmaf(ERz[kk], e1, o[k]);
        }
      }
      float* xo = XB + z0 * bs + C0 + x;
#pragma unroll
      for (int k = 0; k < W; ++k)
        if (z0 + k < nz) xo[k * bs] = o[k];
    }
    if (h1) {
      geometry(i1, y1);
      if (!staged(s1)) return;
    } else {
      __syncthreads();
    }
    // phase B: x pass of p, accumulated over the chunk; gather of p + 1
    const float* ELx = ERz + hz;
    const float* ERx = ELx + hx;
#pragma unroll
    for (int i = 0; i < NT; ++i) {
      const int t = tid + i * NTH;
      if (t < xtasks) {
        const int xb = zdiv(t, rnz), z = t - xb * nz, x0 = W * xb;
        const float* row = XB + z * bs;
        zpassw<W>(Hw + zpw, rg.z, rg.w, row + x0, acc[i]);
        if (x0 < hx) {
          const float e0 = row[C0];
#pragma unroll
          for (int k = 0; k < W; ++k)
            if (x0 + k < hx) acc[i][k] = fmaf(ELx[x0 + k], e0, acc[i][k]);
        }
        if (x0 + W > nx - hx) {
          const float e1 = row[C0 + nx - 1];
#pragma unroll
          for (int k = 0; k < W; ++k) {
            const int kk = nx - 1 - x0 - k;
            if (kk < hx) acc[i][k] = fmaf(ERx[kk], e1, acc[i][k]);
          }
        }
      }
    }
    if (h1) gather(s1, hb ^ 1);
    if (!h1 || i1 != i0) {  // p ends its item: partial view of the chunk, part[slot][ch][z][x]
      const int slot = slot_of(i0), ch = i0 - slot * a.nchunks;
      float* out = a.part + ((size_t)slot * a.nchunks + ch) * nz * nx;
#pragma unroll
      for (int i = 0; i < NT; ++i) {
        const int t = tid + i * NTH;
        if (t < xtasks) {
          const int xb = zdiv(t, rnz), z = t - xb * nz;
          float* o = out + (size_t)z * nx + W * xb;
#pragma unroll
          for (int k = 0; k < W; k += 4) st4(o + k, make_float4(acc[i][k], acc[i][k + 1], acc[i][k + 2], acc[i][k + 3]));
        }
#pragma unroll
        for (int k = 0; k < W; ++k) acc[i][k] = 0.f;
      }
    }
    if (!h1) break;
    __syncthreads();
    refill(s1);
    i0 = i1;
    y0 = y1;
    next(i1, y1);
    hb ^= 1;
    s1 = nsf > 1 ? s1 ^ 1 : 0;
  }
}

// ------------------------------------------------------------------------
// k_zadj<NT, NTH, W>: adjoint convolution (tasks of W outputs); work items (slot, depth chunk), the
// block's planes walked in sequence.  Plane p's adjoint weights and folds are
// bulk-copied three planes ahead (stage p % 3); its x pass (view rows) writes
// the x-pass buffer WB[p % nwa] and its z pass (WB columns, times the
// attenuation column read by 16-byte global loads at the task start) writes
// T.  One phase between two block barriers runs the z pass of plane p and
// the x pass of plane p + 1, so with two buffers each plane costs one barrier
// (one more where plane p + 1 starts a new item: the view is reloaded; and,
// with one buffer, one between the two passes).  NT only sets how the x
// tasks are interleaved.
template <int NT, int NTH, int W>
__global__ void __launch_bounds__(NTH, 1) k_zadj(ZArgs a) {
  extern __shared__ float4 smem4[];
  const ZGeom& g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz, nzp = g.nzp, hs = g.hs, ts = g.ts;
  float* const base = reinterpret_cast<float*>(smem4);
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(base);  // three barriers
  const int sts = hs + ts + 4;             // one stage: weights, folds, tap ranges (4 ints)
  float* const stage = base + 8;
  float* const VB = stage + 3 * sts;
  float* const WB0 = VB + (size_t)nz * g.bs;
  const size_t wbs = g.nwa > 1 ? (size_t)nx * g.ast : 0;  // offset of the second buffer
  const int tid = threadIdx.x;
  const int nitems = a.nv * a.nchunks;
  const float rnc = 1.0f / a.nchunks;
  auto slot_of = [&](int item) { return zdiv(item, rnc); };             // item / nchunks (items < 2^20)
  auto chunk_of = [&](int item) { return item - zdiv(item, rnc) * a.nchunks; };
  auto issue = [&](int item, int y, int s) {  // one thread
    const int sl = slot_of(item), v = a.vidx[sl], set = a.viewset[v];
    float* st = stage + s * sts;
    fence_proxy_async();
    mbar_expect(&bar[s], (unsigned)(sts * sizeof(float)));
    bulk_copy(&bar[s], st, a.H + ((size_t)set * ny + y) * (2 * hs) + hs, (unsigned)(hs * sizeof(float)));
    bulk_copy(&bar[s], st + hs, a.E + ((size_t)set * ny + y) * (2 * ts) + ts, (unsigned)(ts * sizeof(float)));
    bulk_copy(&bar[s], st + hs + ts, a.R + ((size_t)set * ny + y) * 8 + 4, 4u * sizeof(int));
  };
  auto next = [&](int& item, int& y) {
    const int yend = min(ny, chunk_of(item) * a.chunkY + a.chunkY);
    if (y + 1 < yend) {
      ++y;
    } else {
      item += gridDim.x;
      y = chunk_of(item) * a.chunkY;
    }
  };
  // WB rows outside the data rows stay zero
  for (int x = tid / 32; x < g.nwa * nx; x += NTH / 32)
    for (int r = tid & 31; r < g.ast; r += 32)
      if (r < g.R0 || r >= g.R0 + nz) WB0[(size_t)x * g.ast + r] = 0.f;
  // planes p, p + 1, p + 2 and p + 3 (the next to issue)
  int i0 = blockIdx.x, y0 = (blockIdx.x % a.nchunks) * a.chunkY;
  int i1 = i0, y1 = y0;
  next(i1, y1);
  int i2 = i1, y2 = y1;
  next(i2, y2);
  int i3 = i2, y3 = y2;
  next(i3, y3);
  if (tid == 0) {
    mbar_init(&bar[0]);
    mbar_init(&bar[1]);
    mbar_init(&bar[2]);
    if (i0 < nitems) issue(i0, y0, 0);
    if (i1 < nitems) issue(i1, y1, 1);
    if (i2 < nitems) issue(i2, y2, 2);
  }
  __syncthreads();
  if (!(i0 < nitems)) return;
  unsigned pend = (i1 < nitems ? 7u : 1u) & (i2 < nitems ? 7u : 3u);  // copies issued, not yet waited for
  unsigned phases = 0u;                                                  // parity of each barrier's next wait
  auto wait = [&](int s) {
    const bool ok = mbar_wait(&bar[s], (phases >> s) & 1u);
    if (ok) {
      phases ^= 1u << s;
      pend &= ~(1u << s);
    }
    return ok;
  };
  auto give_up = [&]() {  // after a failed wait: flag it, let the copies in flight land
    if (tid == 0) {
      atomicExch(a.err, 1);
      for (int s = 0; s < 3; ++s)
        if ((pend >> s) & 1u) mbar_wait(&bar[s], (phases >> s) & 1u);
    }
  };
  const int nzb = (nz + W - 1) / W, ztasks = nx * nzb, xtasks = nz * (nx / W);
  const int ast = g.ast, bs = g.bs, R0 = g.R0, C0 = g.C0, hz = g.hz, hx = g.hx;
  const float rnx = 1.0f / nx, rnz = 1.0f / nz;
  // the item's view into VB, zero-padded: element e = z bs + c, eight per
  // thread and round with all eight loads issued before the stores
  const float rbs = 1.0f / bs;
  auto load_view = [&](int item) {
    const float* V = a.views + (size_t)slot_of(item) * nz * nx;
    for (int e0 = tid; e0 < nz * bs; e0 += 8 * NTH) {
      float v[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int e = e0 + j * NTH, z = zdiv(e, rbs), c = e - z * bs;
        v[j] = (e < nz * bs && c >= C0 && c < C0 + nx) ? V[z * nx + c - C0] : 0.f;
      }
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (e0 + j * NTH < nz * bs) VB[e0 + j * NTH] = v[j];
    }
  };
  // x pass of the plane whose stage is st: task (z, x block) -> WB column x, row R0 + z
  auto xpass = [&](const float* st, float* WB, int item, int y) {
    const int2 rg = *reinterpret_cast<const int2*>(st + hs + ts + 2);  // x-pass tap range
    const float* ax = st + g.zpw;     // adjoint x weights (shifted)
    const float* cLx = st + hs;       // folds
    const float* cRx = cLx + hx;
#pragma unroll
    for (int i = 0; i < NT; ++i)
      for (int t = tid + i * NTH; t < xtasks; t += NT * NTH) {
        const int xb = zdiv(t, rnz), z = t - xb * nz, x0 = W * xb;
        const float* row = VB + z * bs;
        float o[W];
#pragma unroll
        for (int k = 0; k < W; ++k) o[k] = 0.f;
        zpassw<W>(ax, rg.x, rg.y, row + x0, o);
        if (x0 == 0)
          o[0] += zfold(cLx, row + C0, 1, hx);
        if (x0 + W == nx)
          o[W - 1] += zfold(cRx, row + C0 + nx - 1, -1, hx);
        float* w = WB + x0 * ast + R0 + z;
#pragma unroll
        for (int k = 0; k < W; ++k) w[k * ast] = o[k];
      }
  };
  // z pass of plane (item, y), stage st: task (x, z block) -> T column (x, y) of the slot
  auto zpass = [&](const float* st, const float* WB, int item, int y) {
    const int slot = slot_of(item), v = a.vidx[slot];
    const int2 rg = *reinterpret_cast<const int2*>(st + hs + ts);  // z-pass tap range
    const float* az = st;             // adjoint z weights (shifted)
    const float* cLz = st + hs + 2 * hx;
    const float* cRz = cLz + hz;
    const float* attv = a.att + (((size_t)v * ny + y) * nx) * nzp;
    float* Tp = a.T + (((size_t)slot * ny + y) * nx) * nzp;
    for (int t = tid; t < ztasks; t += NTH) {
      // lanes on consecutive columns: conflict-free shared windows (lanes
      // walking down a column, which coalesces the global accesses, measured
      // slower: 2- to 3-way bank conflicts and folds in every warp)
      const int zb = zdiv(t, rnx), x = t - zb * nx, z0 = W * zb;
      float4 at[W / 4];
#pragma unroll
      for (int k = 0; k < W / 4; ++k) at[k] = ld4(attv + x * nzp + z0 + 4 * k);
      const float* col = WB + x * ast;
      float o[W];
#pragma unroll
      for (int k = 0; k < W; ++k) o[k] = 0.f;
      zpassw<W>(az, rg.x, rg.y, col + z0, o);
      if (z0 == 0)
        o[0] += zfold(cLz, col + R0, 1, hz);
      if (z0 <= nz - 1 && nz - 1 < z0 + W) {
        const int kz = nz - 1 - z0;
        const float s = zfold(cRz, col + R0 + nz - 1, -1, hz);
#pragma unroll
        for (int k = 0; k < W; ++k)
          if (k == kz) o[k] += s;
      }
      float* dst = Tp + x * nzp + z0;
#pragma unroll
      for (int k = 0; k < W / 4; ++k)
        st4(dst + 4 * k, make_float4(__fmul_rn(at[k].x, o[4 * k]), __fmul_rn(at[k].y, o[4 * k + 1]),
                                     __fmul_rn(at[k].z, o[4 * k + 2]), __fmul_rn(at[k].w, o[4 * k + 3])));
    }
  };
  // prologue: the first view, the stages of p and p + 1, the x pass of p
  load_view(i0);
  {
    bool ok = wait(0);
    if (i1 < nitems) ok = wait(1) && ok;
    if (__syncthreads_or(!ok)) {
      give_up();
      return;
    }
  }
  xpass(stage, WB0, i0, y0);
  __syncthreads();
  int s = 0, w = 0;  // stage and x-pass buffer of plane p
  for (;;) {
    const bool h1 = i1 < nitems, h2 = i2 < nitems;
    const int s1 = s == 2 ? 0 : s + 1;
    const bool newv = h1 && slot_of(i1) != slot_of(i0);
    if (newv) load_view(i1);  // the last reader of VB (the x pass of p) finished before the barrier
    zpass(stage + s * sts, WB0 + w * wbs, i0, y0);
    if (h1) {
      if (newv || g.nwa == 1) __syncthreads();  // uniform
      xpass(stage + s1 * sts, WB0 + (w ^ 1) * wbs, i1, y1);
    }
    bool ok = true;
    if (h2) ok = wait(s1 == 2 ? 0 : s1 + 1);
    if (__syncthreads_or(!ok)) {
      give_up();
      return;
    }
    if (!h1) break;
    if (i3 < nitems) {  // stage s is free again: plane p + 3
      if (tid == 0) issue(i3, y3, s);
      pend |= 1u << s;
    }
    i0 = i1;
    y0 = y1;
    i1 = i2;
    y1 = y2;
    i2 = i3;
    y2 = y3;
    next(i3, y3);
    s = s1;
    w ^= 1;
  }
}

// ------------------------------------------------------------------------
// k_zrot_adj<ZPL, RB>: two 8-lane groups of a warp own image column p = (j1, j2)
// (grid-stride), lane l of a group the z pairs 2 l + 16 q, q < ZPL / 2 (nzp =
// 8 ZPL): 64 contiguous bytes per group and 8-byte load.  The first group
// sums the even slots, the second the odd ones; a shuffle adds the two
// partial sums (a fixed order).  Per slot, lane l of a group evaluates
// candidate l (and every lane candidate 8) and the group shares the nine by
// shuffles, summing them in the order 0..8.  For
// every slot, the rotated-grid points (x, y) whose bilinear footprint contains
// (j1, j2) -- those with floor(s1) in {j1-1, j1} and floor(s2) in {j2-1, j2}
// -- lie within |cos| + |sin| of the inverse-rotated pixel centre, so the
// candidates are at most 3 x 3 points; each is tested with the forward's own
// position arithmetic and weighted with the forward's weight product.
// RB = 0: a hit candidate's loads are issued under a branch on its offset,
// so the candidates' load latencies follow one another.  RB > 0: the
// candidates go in rounds of RB whose loads are all issued (predicated off
// for misses, which then read zero) before the round's FMAs, so up to
// RB x ZPL / 2 loads per lane are in flight; a miss adds fmaf(0, 0, acc) ==
// acc, so both forms give the same bits.
// Epilogue (IZ layout): v = acc (+ prev); mode 1: zeros -> +Inf; mode 2:
// v = x * (v / asum); out = v (z < nz only; out may be prev or x).
template <int ZPL, int RB>
__global__ void __launch_bounds__(256, (ZPL <= 14 ? 4 : 2)) k_zrot_adj(ZGeom g, const float* __restrict__ T,
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
    float2 acc[ZPL / 2];
#pragma unroll
    for (int q = 0; q < ZPL / 2; ++q) acc[q] = make_float2(0.f, 0.f);
    // every lane runs the same number of rounds (the shuffles need them all)
    for (int s0 = 0; s0 < nv; s0 += 2) {
      const bool live = s0 + half < nv;
      const int s = live ? s0 + half : s0;
      const float4 r = rot[vidx[s]];
      const float cs = r.x, sn = r.y;
      const float d1 = fj1 - c0, d2 = fj2 - c0;
      const float xc = c0 + cs * d1 + sn * d2, yc = c0 - sn * d1 + cs * d2;
      const float rr = fabsf(cs) + fabsf(sn) + 0.01f;
      const int xlo = max(0, (int)ceilf(xc - rr)), xhi = min(nx - 1, (int)floorf(xc + rr));
      const int ylo = max(0, (int)ceilf(yc - rr)), yhi = min(ny - 1, (int)floorf(yc + rr));
      const float* Ts = T + (size_t)s * ny * nx * nzp + 2 * lane;
      // candidate c = 3 i + k (x offset i, y offset k): weight and column
      // offset (-1: no footprint), with the forward's own operations
      auto cand = [&](int c, float& w, int& o) {
        const int i = (c * 11) >> 5, k = c - 3 * i;  // c / 3 for c <= 8
        const int xx = min(xlo + i, nx - 1), yy = min(ylo + k, ny - 1);
        const float di = __fsub_rn((float)xx, c0), dj = __fsub_rn((float)yy, c0);
        const float s1 = __fadd_rn(c0, __fsub_rn(__fmul_rn(cs, di), __fmul_rn(sn, dj)));
        const float s2 = __fadd_rn(c0, __fadd_rn(__fmul_rn(sn, di), __fmul_rn(cs, dj)));
        const bool ok = live && xlo + i <= xhi && ylo + k <= yhi && s1 >= fj1 - 1.f && s1 < fj1 + 1.f &&
                        s2 >= fj2 - 1.f && s2 < fj2 + 1.f;
        const float f1 = floorf(s1), f2 = floorf(s2);
        const float t1 = __fsub_rn(s1, f1), t2 = __fsub_rn(s2, f2);
        const float a1 = f1 == fj1 ? __fsub_rn(1.0f, t1) : t1;
        const float a2 = f2 == fj2 ? __fsub_rn(1.0f, t2) : t2;
        w = ok ? __fmul_rn(a1, a2) : 0.f;
        o = ok ? (yy * nx + xx) * nzp : -1;
      };
      // lane l of the group evaluates candidate l, every lane candidate 8;
      // the group shares them by shuffles and sums them in the order c = 0..8
      float wl, w8;
      int ol, o8;
      cand(lane, wl, ol);
      cand(8, w8, o8);
      if constexpr (RB == 0) {
#pragma unroll
        for (int c = 0; c < 9; ++c) {
          const float w = c < 8 ? __shfl_sync(0xffffffffu, wl, c, 8) : w8;
          const int o = c < 8 ? __shfl_sync(0xffffffffu, ol, c, 8) : o8;
          if (o >= 0) {
            const float* tp = Ts + o;
#pragma unroll
            for (int q = 0; q < ZPL / 2; ++q) {
              const float2 t = *reinterpret_cast<const float2*>(tp + 16 * q);
              acc[q].x = fmaf(w, t.x, acc[q].x);
              acc[q].y = fmaf(w, t.y, acc[q].y);
            }
          }
        }
      } else {
#pragma unroll
        for (int c0 = 0; c0 < 9; c0 += RB) {
          float wk[RB];
          float2 tk[RB][ZPL / 2];
#pragma unroll
          for (int k = 0; k < RB; ++k) {
            const int c = c0 + k;
            wk[k] = 0.f;
            if (c < 9) {  // resolved at compile time
              wk[k] = c < 8 ? __shfl_sync(0xffffffffu, wl, c, 8) : w8;
              const int o = c < 8 ? __shfl_sync(0xffffffffu, ol, c, 8) : o8;
              const float* tp = Ts + max(o, 0);
#pragma unroll
              for (int q = 0; q < ZPL / 2; ++q) tk[k][q] = ldg2_if(tp + 16 * q, o >= 0);
            }
          }
#pragma unroll
          for (int k = 0; k < RB; ++k) {
            if (c0 + k < 9) {
#pragma unroll
              for (int q = 0; q < ZPL / 2; ++q) {
                acc[q].x = fmaf(wk[k], tk[k][q].x, acc[q].x);
                acc[q].y = fmaf(wk[k], tk[k][q].y, acc[q].y);
              }
            }
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < ZPL / 2; ++q) {  // even + odd slots
      acc[q].x += __shfl_xor_sync(0xffffffffu, acc[q].x, 8);
      acc[q].y += __shfl_xor_sync(0xffffffffu, acc[q].y, 8);
    }
    if (half || !own) continue;
    const size_t o = ((size_t)(j2 + g.pad) * g.L + j1 + g.pad) * nzp + 2 * lane;
#pragma unroll
    for (int q = 0; q < ZPL / 2; ++q) {
      const float vq[2] = {acc[q].x, acc[q].y};
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const size_t oe = o + 16 * q + e;
        if (2 * lane + 16 * q + e < g.nz) {
          float v = vq[e];
          if (prev) v += prev[oe];
          if (mode == 1 && v == 0.f) v = __int_as_float(0x7f800000);
          if (mode == 2) v = x[oe] * (v / asum[oe]);
          out[oe] = v;
        }
      }
    }
  }
}

}  // namespace spect
