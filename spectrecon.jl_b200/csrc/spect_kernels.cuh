// spect_kernels.cuh -- sm_100a kernels of the SPECT projector hot path.
//
// Forward pass of one group of views (project!, src/project.jl:77-135):
//   k_rot_fwd    rotate image and mu-map slices about z (imrotate! :two,
//                src/rotatez.jl:331-362), depth-scan the rotated mu-map and
//                write P[slot][y][z][x] = exp(-dy*(sum_{j<y} mu_j + mu_y/2)) * R(image)
//                (src/project.jl:103-116).  One CTA per (z slice, view split);
//                slices staged in shared memory.
//   k_conv_fwd2  (conv2.cuh) depth-dependent PSF convolution and depth sum.
//   k_reduce_views  sum of the chunk partials in chunk order (+ fused EM ratio).
// Adjoint pass (backproject!, src/backproject.jl:69-124):
//   k_vspec2, k_conv_adj2 (conv2.cuh) adjoint PSF convolution -> T[slot][y][z][x].
//   k_rot_adj    attenuation weighting and the exact transpose of the
//                bilinear rotation (imrotate_adj! :two, src/rotatez.jl:390-416),
//                atomic-free: rotated-grid points are scattered in 9 passes by
//                lattice class (o1 mod 3, o2 mod 3), inside which footprints
//                are disjoint.  Per-view sums in view order.
//   k_reduce_image  sum of split partials (+ fused EM multiplicative update).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "bulk_copy.cuh"
#include "fft_reg.cuh"


namespace spect {

struct Geom {
  int nx, ny, nz;
  int Npx, Npz, logNpx, logNpz, Hz;  // padded FFT sizes (src/helper.jl:8-12), Hz = Npz/2+1
  int padup, padleft;                // _padup(nx,px), _padleft(nz,pz)
  float dy;
  float c0;                          // rotation centre (nx-1)/2, 0-based unpadded
};

// Per-view rotation: x = cos(2pi - theta), y = sin(2pi - theta) rounded to
// float; z = 1 when theta == 0 mod 2pi (the forward :two shortcut copies).
struct RotPos {
  float cs, sn, c0;
  __device__ __forceinline__ void pos(int i, int j, float& s1, float& s2) const {
    float di = __fsub_rn((float)i, c0), dj = __fsub_rn((float)j, c0);
    float a = __fmul_rn(cs, di), b = __fmul_rn(sn, dj), c = __fmul_rn(sn, di), d = __fmul_rn(cs, dj);
    s1 = __fadd_rn(c0, __fsub_rn(a, b));
    s2 = __fadd_rn(c0, __fadd_rn(c, d));
  }
};

// bilinear sample of a zero-extended n x n slice at output pixel (i, j)
__device__ __forceinline__ float bilinear(const float* __restrict__ s, int n, const RotPos& R, int i, int j) {
  float s1, s2;
  R.pos(i, j, s1, s2);
  float f1 = floorf(s1), f2 = floorf(s2);
  int j1 = (int)f1, j2 = (int)f2;
  float t1 = __fsub_rn(s1, f1), t2 = __fsub_rn(s2, f2);
  float u1 = __fsub_rn(1.0f, t1), u2 = __fsub_rn(1.0f, t2);
  bool x0 = (unsigned)j1 < (unsigned)n, x1 = (unsigned)(j1 + 1) < (unsigned)n;
  bool y0 = (unsigned)j2 < (unsigned)n, y1 = (unsigned)(j2 + 1) < (unsigned)n;
  float a = (x0 && y0) ? s[j1 + j2 * n] : 0.f;
  float b = (x1 && y0) ? s[j1 + 1 + j2 * n] : 0.f;
  float c = (x0 && y1) ? s[j1 + (j2 + 1) * n] : 0.f;
  float d = (x1 && y1) ? s[j1 + 1 + (j2 + 1) * n] : 0.f;
  float v = __fmul_rn(__fmul_rn(u1, u2), a);
  v = __fadd_rn(v, __fmul_rn(__fmul_rn(t1, u2), b));
  v = __fadd_rn(v, __fmul_rn(__fmul_rn(u1, t2), c));
  v = __fadd_rn(v, __fmul_rn(__fmul_rn(t1, t2), d));
  return v;
}

// ------------------------------------------------------------------------
// Attenuation factors of one view on the rotated grid, by depth scan along y
// (src/project.jl:103-113): a(x,y,z) = exp(-dy * (sum_{j<y} mu_j + mu_y/2)),
// mu = R_theta(mumap) (imrotate! :two, with the theta == 0 copy).
// k_atten_build: grid (nz, nsplit), block nx * vpb; writes att[v][y][z][x]
// for every plan view (the per-plan attenuation cache).
template <bool SMEM>
__global__ void __launch_bounds__(1024) k_atten_build(Geom g, const float* __restrict__ mumap,
                                                      const float4* __restrict__ rot, int nview,
                                                      float* __restrict__ att) {
  extern __shared__ float4 smem4[];
  const int nx = g.nx, ny = g.ny, nz = g.nz, z = blockIdx.x;
  const size_t slice = (size_t)nx * ny;
  const float* sm = mumap + (size_t)z * slice;
  if (SMEM) {
    float* ss = reinterpret_cast<float*>(smem4);
    for (int k = threadIdx.x; k < (int)slice; k += blockDim.x) ss[k] = __ldg(sm + k);
    __syncthreads();
    sm = ss;
  }
  const int per = (nview + gridDim.y - 1) / gridDim.y;
  const int v0 = blockIdx.y * per, v1 = min(nview, v0 + per);
  const int vpb = blockDim.x / nx, sub = threadIdx.x / nx, x = threadIdx.x - sub * nx;
  if (sub >= vpb) return;
  const float mdy = -g.dy;
  for (int v = v0 + sub; v < v1; v += vpb) {
    const float4 r = rot[v];
    RotPos R{r.x, r.y, g.c0};
    const bool ident = r.z != 0.f;
    float prefix = 0.f;
    float* out = att + ((size_t)v * ny * nz + z) * nx + x;
    for (int y = 0; y < ny; ++y) {
      float m = ident ? sm[x + y * nx] : bilinear(sm, nx, R, x, y);
      float e = __fadd_rn(prefix, __fmul_rn(0.5f, m));
      out[(size_t)y * nz * nx] = expf(__fmul_rn(e, mdy));
      prefix = __fadd_rn(prefix, m);
    }
  }
}

// k_rot_fwd: grid (nz, nsplit), block nx * vpb threads.
// P[slot][y][z][x] = a(x,y,z) * R_theta(image)(x,y,z) for the launch's slots.
// CACHED: a read from the attenuation cache att[view][y][z][x]; otherwise
// the rotated mu-map is scanned here (both slices staged in shared memory
// when SMEM).
template <bool SMEM, bool CACHED>
__global__ void __launch_bounds__(1024) k_rot_fwd(Geom g, const float* __restrict__ image,
                                                  const float* __restrict__ mumap, const float* __restrict__ att,
                                                  const float4* __restrict__ rot, const int* __restrict__ vidx, int nv,
                                                  float* __restrict__ P) {
  extern __shared__ float4 smem4[];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int z = blockIdx.x;
  const size_t slice = (size_t)nx * ny;
  const float* img = image + (size_t)z * slice;
  const float* mu = mumap + (size_t)z * slice;
  if (SMEM) {
    float* si = reinterpret_cast<float*>(smem4);
    float* sm = si + slice;
    for (int k = threadIdx.x; k < (int)slice; k += blockDim.x) {
      si[k] = __ldg(img + k);
      if (!CACHED) sm[k] = __ldg(mu + k);
    }
    __syncthreads();
    img = si;
    mu = sm;
  }
  const int per = (nv + gridDim.y - 1) / gridDim.y;
  const int s0 = blockIdx.y * per, s1 = min(nv, s0 + per);
  const int vpb = blockDim.x / nx;
  const int sub = threadIdx.x / nx, x = threadIdx.x - sub * nx;
  if (sub >= vpb) return;
  const float mdy = -g.dy;
  for (int s = s0 + sub; s < s1; s += vpb) {
    const int v = vidx[s];
    const float4 r = rot[v];
    RotPos R{r.x, r.y, g.c0};
    const bool ident = r.z != 0.f;
    float prefix = 0.f;
    float* out = P + ((size_t)s * ny * nz + z) * nx + x;
#pragma unroll 8
    for (int y = 0; y < ny; ++y) {
      const float f = ident ? img[x + y * nx] : bilinear(img, nx, R, x, y);
      float a;
      if (CACHED) {
        // the convolution kernel applies the cached attenuation on load
        out[(size_t)y * nz * nx] = f;
        continue;
      } else {
        const float m = ident ? mu[x + y * nx] : bilinear(mu, nx, R, x, y);
        // exp(-dy * (sum_{j<y} mu_j + mu_y/2))  (src/project.jl:103-113)
        const float e = __fadd_rn(prefix, __fmul_rn(0.5f, m));
        a = expf(__fmul_rn(e, mdy));
        prefix = __fadd_rn(prefix, m);
      }
      out[(size_t)y * nz * nx] = __fmul_rn(f, a);
    }
  }
}

// ------------------------------------------------------------------------
// k_reduce_views: out[slot] = sum_c part[slot][c]; with EM, out = y/(sum+bg)
__global__ void k_reduce_views(const float* __restrict__ part, int nv, int nchunks, int nxz,
                               float* __restrict__ out, const float* __restrict__ y, const float* __restrict__ bg,
                               const int* __restrict__ vidx) {
  const size_t n = (size_t)nv * nxz;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    size_t slot = k / nxz, e = k - slot * nxz;
    const float* p = part + slot * nchunks * nxz + e;
    float sacc = p[0];
    for (int c = 1; c < nchunks; ++c) sacc += p[(size_t)c * nxz];
    if (y) {
      size_t src = (size_t)vidx[slot] * nxz + e;
      sacc = y[src] / (sacc + bg[src]);
    }
    out[k] = sacc;
  }
}

// ------------------------------------------------------------------------
// ------------------------------------------------------------------------
// Transpose of the bilinear sampling for one lattice class (c1, c2) of the
// rotated-grid rows [r0, r0 + nr): point (o1, o2), o1 = c1 mod 3, o2 = c2
// mod 3, with value S[(o2 - r0) * nx + o1], adds its four bilinear weights
// (exactly those of bilinear()) into acc rows [ya, yb) (acc row stride as
// >= nx + 2).  acc must be guarded: rows ya-1 and yb and columns -1 and nx
// addressable (the padding of the neighbouring rows serves as columns).
// Inside a class two footprints are >= 3/sqrt 2 > 2 pixels apart, so no two
// points of the pass touch the same accumulator: each thread keeps two
// points in flight and the block synchronises only between passes.

// thread walk over the columns o1 = c1, c1 + 3, ... of one class: npt
// columns; the block steps (dq rows, dm columns) at a time; this thread
// starts at (q0, m0).  Computed once per kernel (runtime divisions).
struct ClassCols {
  int npt, dq, dm, q0, m0;
};
__device__ __forceinline__ ClassCols class_cols(int nx, int c1) {
  ClassCols w;
  w.npt = (nx - c1 + 2) / 3;
  w.dq = blockDim.x / w.npt;
  w.dm = blockDim.x - w.dq * w.npt;
  w.q0 = threadIdx.x / w.npt;
  w.m0 = threadIdx.x - w.q0 * w.npt;
  return w;
}

// rotated positions from per-view tables: PA[o1] = (cs (o1 - c0), sn (o1 - c0)),
// PB[o2] = (sn (o2 - c0), cs (o2 - c0)), the products of RotPos::pos rounded
// the same way, so s = c0 + (PA.x - PB.x, PA.y + PB.y) is bit-identical
struct PosTab {
  const float2* PA;
  const float2* PB;
};
__device__ __forceinline__ void build_postab(const RotPos& R, int nx, int ny, float2* PA, float2* PB) {
  for (int e = threadIdx.x; e < nx + ny; e += blockDim.x) {
    const int o = e < nx ? e : e - nx;
    const float d = __fsub_rn((float)o, R.c0);
    if (e < nx) PA[o] = make_float2(__fmul_rn(R.cs, d), __fmul_rn(R.sn, d));
    else PB[o] = make_float2(__fmul_rn(R.sn, d), __fmul_rn(R.cs, d));
  }
}

// PTAB: positions from a PosTab (else RotPos::pos)
template <bool GUARD, bool PTAB>
__device__ __forceinline__ void scatter_class(const RotPos R, const PosTab PT, const float* S, int nx, int r0,
                                              int nr, int c1, int c2, const ClassCols cw, float* acc, int as,
                                              int ya, int yb) {
  const int o2f = r0 + (c2 - r0 % 3 + 3) % 3;
  const int nrow = o2f < r0 + nr ? (r0 + nr - 1 - o2f) / 3 + 1 : 0;
  const int npt = cw.npt, dq = cw.dq, dm = cw.dm;
  int q = cw.q0, m = cw.m0;
  auto step = [&](int& qq, int& mm) {
    qq += dq;
    mm += dm;
    if (mm >= npt) {
      mm -= npt;
      ++qq;
    }
  };
  while (q < nrow) {
    int qb = q, mb = m;
    step(qb, mb);
    const bool hasb = qb < nrow;
    float w[2][4], val[2], old[2][4];
    int base[2];
    bool ok[2], tk[2][4];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int qq = k ? qb : q, mm = k ? mb : m;
      const int o2 = o2f + 3 * qq, o1 = c1 + 3 * mm;
      const bool act = k ? hasb : true;
      val[k] = act ? S[(o2 - r0) * nx + o1] : 0.f;
      float s1, s2;
      if (PTAB) {
        // an inactive second point may lie past the last row: read row r0
        const float2 pa = PT.PA[o1], pb = PT.PB[act ? o2 : r0];
        s1 = __fadd_rn(R.c0, __fsub_rn(pa.x, pb.x));
        s2 = __fadd_rn(R.c0, __fadd_rn(pa.y, pb.y));
      } else {
        R.pos(o1, o2, s1, s2);
      }
      const float f1 = floorf(s1), f2 = floorf(s2);
      const int j1 = (int)f1, j2 = (int)f2;
      const float t1 = __fsub_rn(s1, f1), t2 = __fsub_rn(s2, f2);
      const float u1 = __fsub_rn(1.0f, t1), u2 = __fsub_rn(1.0f, t2);
      // GUARD: footprint {j1, j1+1} x {j2, j2+1} inside the guarded
      // accumulator (columns -1..nx, rows ya-1..yb); taps outside the image
      // land in guard cells, which are never read back.  Otherwise each tap
      // is checked against the image.
      ok[k] = act && (unsigned)(j1 + 1) <= (unsigned)nx && (unsigned)(j2 + 1 - ya) <= (unsigned)(yb - ya);
      if (!GUARD) {
        tk[k][0] = j1 >= 0 && j2 >= ya;
        tk[k][1] = j1 + 1 < nx && j2 >= ya;
        tk[k][2] = j1 >= 0 && j2 + 1 < yb;
        tk[k][3] = j1 + 1 < nx && j2 + 1 < yb;
      }
      w[k][0] = __fmul_rn(u1, u2);
      w[k][1] = __fmul_rn(t1, u2);
      w[k][2] = __fmul_rn(u1, t2);
      w[k][3] = __fmul_rn(t1, t2);
      base[k] = j1 + (j2 - ya) * as;
    }
    const int off[4] = {0, 1, 0, 1};
#pragma unroll
    for (int k = 0; k < 2; ++k)
      if (ok[k]) {
#pragma unroll
        for (int t = 0; t < 4; ++t)
          old[k][t] = (GUARD || tk[k][t]) ? acc[base[k] + off[t] + (t >> 1) * as] : 0.f;
      }
#pragma unroll
    for (int k = 0; k < 2; ++k)
      if (ok[k]) {
#pragma unroll
        for (int t = 0; t < 4; ++t)
          if (GUARD || tk[k][t])
            acc[base[k] + off[t] + (t >> 1) * as] = __fadd_rn(old[k][t], __fmul_rn(w[k][t], val[k]));
      }
    q = qb;
    m = mb;
    step(q, m);
  }
}

// guarded accumulator row stride: at least nx + 2 (the padding of a row
// holds guard columns nx and -1 of the next row), 5 mod 32 so that the taps
// of a warp's points along a rotated line spread over the banks
__host__ __device__ constexpr int acc_stride(int nx) { return nx + 2 + ((5 - (nx + 2)) % 32 + 32) % 32; }
// floats of a guarded accumulator of `rows` rows (guard rows above and
// below), rounded to 16 bytes; its element (0, 0) is at offset as + 1
__host__ __device__ constexpr int acc_floats(int rows, int as) { return ((rows + 2) * as + 3) & ~3; }

// k_rot_adj: grid (nz, nsplit), block kRotAdjThreads.  Accumulates
// sum_s R'(a_s .* T_s) for the slots of this split into acc (shared or the
// global per-CTA buffer) and adds/writes it into imgpart[split][z][:][:].
// CACHED: a_s from the attenuation cache; otherwise rotated mu-map + depth
// scan per view (imrotate! of the mu-map and the attenuation of
// src/backproject.jl:77-109).
constexpr int kRotAdjThreads = 512;

template <bool CACHED>
__global__ void __launch_bounds__(kRotAdjThreads, 1) k_rot_adj(Geom g, const float* __restrict__ T,
                                                                const float* __restrict__ mumap,
                                                                const float* __restrict__ att,
                                                                const float4* __restrict__ rot,
                                                                const int* __restrict__ vidx, int nv,
                                                                float* __restrict__ imgpart, int accumulate,
                                                                int use_smem, float* __restrict__ gscr) {
  extern __shared__ float4 smem4[];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int z = blockIdx.x, split = blockIdx.y;
  const int slice = nx * ny;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  float* acc;
  float* S;
  float* segsum;
  const int nseg = max(1, (int)blockDim.x / nx);
  if (use_smem) {
    acc = reinterpret_cast<float*>(smem4);
    S = acc + slice;
    segsum = S + slice;
  } else {
    size_t cta = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
    acc = gscr + cta * (2 * (size_t)slice + (size_t)nseg * nx);
    S = acc + slice;
    segsum = S + slice;
  }
  float* outp = imgpart + ((size_t)split * nz + z) * slice;
  const ClassCols cw0 = class_cols(nx, 0), cw1 = class_cols(nx, 1), cw2 = class_cols(nx, 2);
  for (int y = warp; y < ny; y += nwarps)
    for (int x = lane; x < nx; x += 32) acc[y * nx + x] = accumulate ? outp[y * nx + x] : 0.f;
  const float* mu = mumap + (size_t)z * slice;
  const int per = (nv + gridDim.y - 1) / gridDim.y;
  const int s0 = split * per, s1 = min(nv, s0 + per);
  const float mdy = -g.dy;
  const int seglen = (ny + nseg - 1) / nseg;
  const int myseg = threadIdx.x / nx, o1s = threadIdx.x - myseg * nx;
  for (int s = s0; s < s1; ++s) {
    const int v = vidx[s];
    const float4 r = rot[v];
    RotPos R{r.x, r.y, g.c0};
    const bool ident = r.z != 0.f;
    __syncthreads();
    if (CACHED) {
      // S = a .* T on the rotated grid (coalesced rows of x)
      const float* av = att + ((size_t)v * ny * nz + z) * nx;
      const float* tv = T + ((size_t)s * ny * nz + z) * nx;
      for (int y = warp; y < ny; y += nwarps)
        for (int x = lane; x < nx; x += 32) {
          const size_t o = (size_t)y * nz * nx + x;
          S[y * nx + x] = __fmul_rn(__ldg(av + o), __ldg(tv + o));
        }
    } else {
      // 1) rotated mu-map of this view on the rotated grid (forward sampling)
      for (int y = warp; y < ny; y += nwarps)
        for (int x = lane; x < nx; x += 32) S[y * nx + x] = ident ? __ldg(mu + y * nx + x) : bilinear(mu, nx, R, x, y);
      __syncthreads();
      // 2) depth scan along y per column x, attenuation, times T
      if (myseg < nseg) {
        const int ya = myseg * seglen, yb = min(ny, ya + seglen);
        float sum = 0.f;
        for (int y = ya; y < yb; ++y) sum = __fadd_rn(sum, S[y * nx + o1s]);
        segsum[myseg * nx + o1s] = sum;
      }
      __syncthreads();
      if (myseg < nseg) {
        const int ya = myseg * seglen, yb = min(ny, ya + seglen);
        float prefix = 0.f;
        for (int q = 0; q < myseg; ++q) prefix = __fadd_rn(prefix, segsum[q * nx + o1s]);
        const float* Tc = T + ((size_t)s * ny * nz + z) * nx + o1s;
        for (int y = ya; y < yb; ++y) {
          float m = S[y * nx + o1s];
          float e = __fadd_rn(prefix, __fmul_rn(0.5f, m));
          float at = expf(__fmul_rn(e, mdy));
          S[y * nx + o1s] = __fmul_rn(at, __ldg(Tc + (size_t)y * nz * nx));
          prefix = __fadd_rn(prefix, m);
        }
      }
    }
    __syncthreads();
    // 3) transpose of the bilinear sampling: 9 lattice classes (o1 mod 3,
    //    o2 mod 3); inside a class the 2x2 footprints of two points are >= 2.1
    //    pixels apart (|Rot (3a,3b)|_inf >= 3/sqrt 2), so they never overlap
    for (int cls = 0; cls < 9; ++cls) {
      const int c1 = cls % 3;
      scatter_class<false, false>(R, PosTab{}, S, nx, 0, ny, c1, cls / 3, c1 == 0 ? cw0 : c1 == 1 ? cw1 : cw2, acc,
                                  nx, 0, ny);
      __syncthreads();
    }
  }
  __syncthreads();
  for (int y = warp; y < ny; y += nwarps)
    for (int x = lane; x < nx; x += 32) outp[y * nx + x] = acc[y * nx + x];
}

// k_rot_adj_stream: persistent form of the cached adjoint rotation for
// premultiplied slices (the adjoint convolution applied a_s).  Work items are
// (slice z, view split) pairs, item = split * nz + z, taken by the blocks in
// grid-stride order; each block walks the sequence of (item, slot) of its
// items and bulk-copies the rows of the next slot's slice (which may belong
// to its next item) into the second of two shared buffers while it scatters
// the current one, so only the block's very first copy is waited on.  The
// accumulator (rows padded to acc_stride) is written to imgpart[split][z] at
// the end of each item and re-initialised for the next.
__global__ void __launch_bounds__(kRotAdjThreads, 1) k_rot_adj_stream(Geom g, const float* __restrict__ T,
                                                                       const float4* __restrict__ rot,
                                                                       const int* __restrict__ vidx, int nv,
                                                                       int nsplit, float* __restrict__ imgpart,
                                                                       int accumulate, int* err) {
  extern __shared__ float4 smem4[];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int slice = nx * ny;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const int as = acc_stride(nx);
  const ClassCols cw0 = class_cols(nx, 0), cw1 = class_cols(nx, 1), cw2 = class_cols(nx, 2);
  float* const acc = reinterpret_cast<float*>(smem4) + as + 1;  // guarded (acc_floats)
  float* const Sb0 = reinterpret_cast<float*>(smem4) + acc_floats(ny, as);
  float* const Sb1 = Sb0 + slice;
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(Sb1 + slice);
  float2* const PA = reinterpret_cast<float2*>(bar + 2);  // position tables (nx + ny)
  float2* const PB = PA + nx;
  const int nitems = nz * nsplit;
  const int per = (nv + nsplit - 1) / nsplit;
  // next (item, slot) of this block after (it, s); it >= nitems when done
  auto next = [&](int& it, int& s) {
    if (s + 1 < min(nv, (it / nz) * per + per)) {
      ++s;
      return;
    }
    for (it += gridDim.x; it < nitems; it += gridDim.x) {
      s = (it / nz) * per;
      if (s < nv) return;
    }
  };
  auto issue = [&](int it, int sl, int b) {  // warp 0
    const int z = it % nz;
    if (lane == 0) {
      fence_proxy_async();
      mbar_expect(&bar[b], (unsigned)(slice * sizeof(float)));
    }
    __syncwarp();
    fence_proxy_async();
    float* dst = b ? Sb1 : Sb0;
    for (int y = lane; y < ny; y += 32)
      bulk_copy(&bar[b], dst + (size_t)y * nx, T + (((size_t)sl * ny + y) * nz + z) * nx,
                (unsigned)(nx * sizeof(float)));
  };
  if (threadIdx.x == 0) {
    mbar_init(&bar[0]);
    mbar_init(&bar[1]);
  }
  // splits without slots still own a partial image: zero it on a first group
  if (!accumulate)
    for (int e = blockIdx.x; e < nitems; e += gridDim.x)
      if ((e / nz) * per >= nv) {
        float* o = imgpart + ((size_t)(e / nz) * nz + e % nz) * slice;
        for (int k = threadIdx.x; k < slice; k += blockDim.x) o[k] = 0.f;
      }
  __syncthreads();
  int it = blockIdx.x - (int)gridDim.x, s = nv;  // advance to the first (item, slot)
  next(it, s);
  if (warp == 0 && it < nitems) issue(it, s, 0);
  unsigned phases = 0u;  // bit b: parity of buffer b's next phase
  int b = 0, cur = -1;
  while (it < nitems) {
    const int z = it % nz, split = it / nz;
    float* outp = imgpart + ((size_t)split * nz + z) * slice;
    if (it != cur) {
      // same (y, x) mapping as the write-out below: no barrier needed
      for (int y = warp; y < ny; y += nwarps)
        for (int x = lane; x < nx; x += 32) acc[y * as + x] = accumulate ? outp[y * nx + x] : 0.f;
      cur = it;
    }
    const unsigned par = (phases >> b) & 1u;
    if (__syncthreads_or(!mbar_wait(&bar[b], par))) {
      if (threadIdx.x == 0) {
        atomicExch(err, 1);
        mbar_wait(&bar[b], par);
      }
      return;
    }
    phases ^= 1u << b;
    int it2 = it, s2 = s;
    next(it2, s2);
    if (warp == 0 && it2 < nitems) issue(it2, s2, b ^ 1);
    const float4 r = rot[vidx[s]];
    const RotPos R{r.x, r.y, g.c0};
    const float* S = b ? Sb1 : Sb0;
    build_postab(R, nx, ny, PA, PB);
    __syncthreads();
    for (int cls = 0; cls < 9; ++cls) {
      const int c1 = cls % 3;
      scatter_class<true, true>(R, PosTab{PA, PB}, S, nx, 0, ny, c1, cls / 3, c1 == 0 ? cw0 : c1 == 1 ? cw1 : cw2,
                                acc, as, 0, ny);
      __syncthreads();
    }
    if (it2 != it) {
      for (int y = warp; y < ny; y += nwarps)
        for (int x = lane; x < nx; x += 32) outp[y * nx + x] = acc[y * as + x];
    }
    b ^= 1;
    it = it2;
    s = s2;
  }
}

// k_rot_adj_band: the adjoint rotation for slices too large for shared
// memory.  grid (nz, nsplit, nband): each block owns a band of output rows of
// slice z (its accumulator stays in shared memory) and streams the
// premultiplied slices T of its slots through two shared buffers of
// kRotBandRows rows (bulk copies).  Chunks of rows whose rotated positions
// cannot reach the band are skipped.  The 9-class scatter is that of
// k_rot_adj, restricted to taps inside the band.
constexpr int kRotBandRows = 32;

__global__ void __launch_bounds__(kRotAdjThreads, 1) k_rot_adj_band(Geom g, const float* __restrict__ T,
                                                                     const float4* __restrict__ rot,
                                                                     const int* __restrict__ vidx, int nv,
                                                                     float* __restrict__ imgpart, int accumulate,
                                                                     int nband, int* err) {
  extern __shared__ float4 smem4[];
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int z = blockIdx.x, split = blockIdx.y;
  const int rows = (ny + nband - 1) / nband;
  const int ya = blockIdx.z * rows, yb = min(ny, ya + rows);
  if (ya >= yb) return;  // uniform over the block
  constexpr int CH = kRotBandRows;
  const int nch = (ny + CH - 1) / CH;
  const int as = acc_stride(nx);
  const ClassCols cw0 = class_cols(nx, 0), cw1 = class_cols(nx, 1), cw2 = class_cols(nx, 2);
  float* const acc = reinterpret_cast<float*>(smem4) + as + 1;  // guarded (acc_floats)
  float* const Sb0 = reinterpret_cast<float*>(smem4) + acc_floats(rows, as);
  float* const Sb1 = Sb0 + (size_t)CH * nx;
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(Sb1 + (size_t)CH * nx);
  float2* const PA = reinterpret_cast<float2*>(bar + 2);  // position tables (nx + ny)
  float2* const PB = PA + nx;
  int s_tab = -1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* outp = imgpart + (((size_t)split * nz + z) * ny + ya) * nx;
  const int nwarps = blockDim.x >> 5;
  for (int y = warp; y < yb - ya; y += nwarps)
    for (int x = lane; x < nx; x += 32) acc[y * as + x] = accumulate ? outp[y * nx + x] : 0.f;
  const int per = (nv + gridDim.y - 1) / gridDim.y;
  const int s0 = split * per, s1 = min(nv, s0 + per);
  const float c0 = g.c0;
  // can rows [c*CH, c*CH + CH) of slot s reach rows [ya, yb)?  s2 is affine
  // in (o1, o2): bound it by the corners, with a one-pixel margin
  auto reach = [&](int s, int c) -> bool {
    const float4 r = rot[vidx[s]];
    const float r0 = (float)(c * CH), r1 = (float)(min(ny, c * CH + CH) - 1);
    const float a0 = r.y * (0.f - c0), a1 = r.y * ((float)(nx - 1) - c0);
    const float b0 = r.x * (r0 - c0), b1 = r.x * (r1 - c0);
    const float lo = c0 + fminf(a0, a1) + fminf(b0, b1), hi = c0 + fmaxf(a0, a1) + fmaxf(b0, b1);
    return hi > (float)ya - 2.f && lo < (float)yb + 1.f;
  };
  auto next = [&](int& s, int& c) {
    for (;;) {
      if (++c >= nch) {
        c = 0;
        ++s;
      }
      if (s >= s1 || reach(s, c)) return;
    }
  };
  auto issue = [&](int s, int c, int b) {  // warp 0
    const int r0 = c * CH, nr = min(ny - r0, CH);
    if (lane == 0) {
      fence_proxy_async();
      mbar_expect(&bar[b], (unsigned)(nr * nx * sizeof(float)));
    }
    __syncwarp();
    fence_proxy_async();
    float* dst = b ? Sb1 : Sb0;
    for (int y = lane; y < nr; y += 32)
      bulk_copy(&bar[b], dst + (size_t)y * nx, T + (((size_t)s * ny + r0 + y) * nz + z) * nx,
                (unsigned)(nx * sizeof(float)));
  };
  if (threadIdx.x == 0) {
    mbar_init(&bar[0]);
    mbar_init(&bar[1]);
  }
  __syncthreads();
  int s = s0, c = -1;
  if (s < s1) next(s, c);
  if (warp == 0 && s < s1) issue(s, c, 0);
  unsigned phases = 0u;  // bit b: parity of buffer b's next phase
  int b = 0;
  while (s < s1) {
    const unsigned par = (phases >> b) & 1u;
    if (__syncthreads_or(!mbar_wait(&bar[b], par))) {
      if (threadIdx.x == 0) {
        atomicExch(err, 1);
        mbar_wait(&bar[b], par);
      }
      return;
    }
    phases ^= 1u << b;
    int sn = s, cn = c;
    next(sn, cn);
    if (warp == 0 && sn < s1) issue(sn, cn, b ^ 1);
    const float4 r = rot[vidx[s]];
    const RotPos R{r.x, r.y, c0};
    const int r0 = c * CH, nr = min(ny - r0, CH);
    const float* S = b ? Sb1 : Sb0;
    if (s != s_tab) {  // new slot: its position tables
      build_postab(R, nx, ny, PA, PB);
      s_tab = s;
      __syncthreads();
    }
    for (int cls = 0; cls < 9; ++cls) {
      const int c1 = cls % 3;
      scatter_class<true, true>(R, PosTab{PA, PB}, S, nx, r0, nr, c1, cls / 3,
                                c1 == 0 ? cw0 : c1 == 1 ? cw1 : cw2, acc, as, ya, yb);
      __syncthreads();
    }
    b ^= 1;
    s = sn;
    c = cn;
  }
  __syncthreads();
  for (int y = warp; y < yb - ya; y += nwarps)
    for (int x = lane; x < nx; x += 32) outp[y * nx + x] = acc[y * as + x];
}

// k_reduce_image: img = sum_split imgpart[split]; EM: x .*= img ./ asum
__global__ void k_reduce_image(const float* __restrict__ imgpart, int nsplit, size_t N, float* __restrict__ out,
                               const float* __restrict__ asum, int em_update, int inf_zero) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < N; k += (size_t)gridDim.x * blockDim.x) {
    float v = imgpart[k];
    for (int s = 1; s < nsplit; ++s) v += imgpart[(size_t)s * N + k];
    if (inf_zero && v == 0.f) v = __int_as_float(0x7f800000);  // asum zeros -> Inf
    if (em_update) out[k] = out[k] * (v / asum[k]);
    else out[k] = v;
  }
}

// psf_gauss on the device (src/psf-gauss.jl:24-55) for planes y in
// [y0, y0 + n): psf[y - y0][j][i] = wx[i] * wz[j], each axis a normalised
// Gaussian exp(-r^2 / (2 sigma^2)), sigma = fwhm / sqrt(log 256), r = -h..h;
// fwhm = 0 gives the Kronecker impulse.  fwhm(y) = start + y * (end - start)
// / (ny - 1) (end exactly at y = ny - 1), in double as the host generator
// (numpy.linspace's rule).  One thread per tap.
__device__ __forceinline__ double gauss_fwhm(int y, int ny, double a, double b) {
  if (ny <= 1) return a;
  return y == ny - 1 ? b : a + y * ((b - a) / (ny - 1));
}
__device__ double gauss_tap(int r, int p, double fwhm) {
  const int h = (p - 1) / 2;
  if (fwhm == 0.0) return r == 0 ? 1.0 : 0.0;
  const double sigma = fwhm / sqrt(log(256.0));
  double s = 0.0;
  for (int i = 0; i < p; ++i) {
    const double q = (double)(-h + i) / sigma;
    s += exp(-0.5 * q * q);
  }
  const double q = (double)r / sigma;
  return exp(-0.5 * q * q) / s;
}
__global__ void k_psf_gauss(float* __restrict__ psf, int y0, int n, int ny, int px, int pz, double x0, double x1,
                            double z0, double z1) {
  const size_t pp = (size_t)px * pz, total = (size_t)n * pp;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
    const int y = y0 + (int)(k / pp);
    const int e = (int)(k % pp), j = e / px, i = e - j * px;
    const double wx = gauss_tap(i - (px - 1) / 2, px, gauss_fwhm(y, ny, x0, x1));
    const double wz = gauss_tap(j - (pz - 1) / 2, pz, gauss_fwhm(y, ny, z0, z1));
    psf[k] = (float)(wx * wz);
  }
}

// ------------------------------------------------------------------------
// PSF spectra: H[set][y][kz][kx] = Re sum_{d,e} h[d,e] w_x^{kx d} w_z^{kz e} / (Npx Npz)
// with h[d,e] = psf[(pz-1)/2+e][(px-1)/2+d], the circularly centred kernel
// (pad2sizezero! + fftshift2!, src/helper.jl:66-80, 111-142).  Double math.
__global__ void k_psf_stage1(const float* __restrict__ psf, int nplanes, int px, int pz, int Npx,
                             const double2* __restrict__ wx, double2* __restrict__ G) {
  // G[pl][e][kx] = sum_d h[d,e] w_x^{(kx*d) mod Npx}
  const size_t n = (size_t)nplanes * pz * Npx;
  const int cx = (px - 1) / 2;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int kx = (int)(k % Npx);
    size_t r = k / Npx;
    int e = (int)(r % pz);
    size_t pl = r / pz;
    const float* row = psf + (pl * pz + e) * px;
    double re = 0, im = 0;
    for (int a = 0; a < px; ++a) {
      int d = a - cx;
      int m = (int)(((long long)kx * d) % Npx);
      if (m < 0) m += Npx;
      double2 w = wx[m];
      double h = (double)row[a];
      re += h * w.x;
      im += h * w.y;
    }
    G[k] = make_double2(re, im);
  }
}

__global__ void k_psf_stage2(const double2* __restrict__ G, int nplanes, int pz, int Npx, int Npz, int Hz,
                             const double2* __restrict__ wz, float* __restrict__ H) {
  const size_t n = (size_t)nplanes * Hz * Npx;
  const int cz = (pz - 1) / 2;
  const double scale = 1.0 / ((double)Npx * Npz);
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int kx = (int)(k % Npx);
    size_t r = k / Npx;
    int kz = (int)(r % Hz);
    size_t pl = r / Hz;
    double re = 0;
    for (int b = 0; b < pz; ++b) {
      int e = b - cz;
      int m = (int)(((long long)kz * e) % Npz);
      if (m < 0) m += Npz;
      double2 w = wz[m], gv = G[(pl * pz + b) * Npx + kx];
      re += gv.x * w.x - gv.y * w.y;
    }
    H[k] = (float)(re * scale);
  }
}

// Hs[pl][c][k1x*CX + lx] in the scrambled orders of the conv kernels
// (conv2.cuh) from H[pl][kz][kx] (kz < Npz/2+1).
__global__ void k_psf_permute(const float* __restrict__ H, int nplanes, int Npx, int Npz, int Hz, int RX, int logCX,
                              int RZ, int logCZ, int Q, float* __restrict__ Hs) {
  const size_t n = (size_t)nplanes * (Q + 1) * Npx;
  const int CX = 1 << logCX, CZ = 1 << logCZ, half = CZ >> 1;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const int pos = (int)(k % Npx);
    const size_t r = k / Npx;
    const int c = (int)(r % (Q + 1));
    const size_t pl = r / (Q + 1);
    const int k1 = pos / CX, l = pos - k1 * CX;
    // lane l, register k1 of the x transform: the 256-point layout of
    // fftx256_fwd, else X[k1 + RX brev(l)]
    const int kx = RX == 8 ? x256_freq(l, k1) : k1 + RX * (logCX ? (int)(__brev(l) >> (32 - logCX)) : 0);
    const float* Hp = H + pl * Hz * Npx;
    float v;
    if (c == 0 || c == Q) {
      float h0 = Hp[kx], hn = (Npz >= 2) ? Hp[(size_t)(Npz / 2) * Npx + kx] : 0.f;
      if (Npz >= 2) v = (c == 0) ? 0.5f * (h0 + hn) : 0.5f * (h0 - hn);
      else v = (c == 0) ? h0 : 0.f;
    } else {
      const int k1z = c / half, lz = 2 * (c - k1z * half);
      const int kz = k1z + RZ * (logCZ ? (int)(__brev(lz) >> (32 - logCZ)) : 0);
      v = Hp[(size_t)kz * Npx + kx];
    }
    Hs[k] = v;
  }
}

}  // namespace spect
