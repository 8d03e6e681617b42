// sconv.cuh -- depth-dependent PSF convolution for separable (rank-1) PSF
// planes, by direct FP32 FMAs (sm_100a).
//
// fft_conv!/fft_conv_adj! (src/fft_convolve.jl:33-130) equal the
// replicate-boundary linear convolution with the centred, point-symmetric
// kernel:  out[x,z] = sum_{d,e} h[d,e] img[clamp(x-d), clamp(z-e)].  When a
// plane's kernel factors as h[d,e] = a[d] b[e] (every psf_gauss plane does,
// up to float rounding of the product), the 2-D convolution is a z pass
// followed by an x pass, each with the clamped (replicated) boundary:
// (nx*nz)*(px+pz) FMAs per plane instead of two 2-D FFTs.  The plan detects
// the factorisation (relative residual <= 1e-6 on every plane) and falls back
// to the FFT kernels otherwise.
//
// Weights per (set, plane), row H[set][y][*] of 2 * hs floats (hs = zp + xp,
// zp = pz rounded up to kSepZB, xp = px rounded up to kSepXB, zero padded):
//   [0, zp)            wz[m] = b[pz-1-m]   forward z pass (reversed factor)
//   [zp, hs)           wx[m] = a[px-1-m]   forward x pass
//   [hs, hs+zp)        b[m]                adjoint z pass (correlation)
//   [hs+zp, 2 hs)      a[m]                adjoint x pass
// so every pass is out[i] = sum_m w[m] line[i + m] over a padded line, with
// the zero weights past the factor length making the padded taps vanish.
//
// Both kernels work in register tiles: a task owns kSepZB (z pass) or kSepXB
// (x pass) consecutive outputs and keeps the inputs it needs in a sliding
// register window; a thread runs its NT x tasks and NZ = (NT+1)/2 z tasks in
// lock step (tasks assigned round-robin, so every warp gets the same work and
// one broadcast load of a block of weights feeds many FMAs).
#pragma once
#include <cuda_runtime.h>

#include "bulk_copy.cuh"

namespace spect {

constexpr int kSepZB = 8;  // z outputs per z-pass task
constexpr int kSepXB = 8;  // x outputs per x-pass task

// launch shapes: NT x-pass tasks per thread, NTH threads per block (one block
// per SM; 640 threads leave at most 102 registers a thread, 1024 threads 64:
// each NT here runs without spills)
struct SepShape {
  int nt, nth;
};
constexpr int kSepNShapes = 9;
constexpr SepShape kSepShapes[kSepNShapes] = {{1, 512}, {2, 512}, {3, 512}, {4, 512}, {1, 640},
                                              {2, 640}, {3, 640}, {1, 1024}, {2, 1024}};

__host__ __device__ constexpr int sep_zp(int pz) { return (pz + kSepZB - 1) / kSepZB * kSepZB; }
__host__ __device__ constexpr int sep_xp(int px) { return (px + kSepXB - 1) / kSepXB * kSepXB; }
// rows of the z-padded buffers (Apad, Wpad): every window read stays inside
__host__ __device__ constexpr int sep_rows(int nz, int pz) {
  return (nz + kSepZB - 1) / kSepZB * kSepZB + sep_zp(pz);
}
// row stride of the x-padded buffers (Bz, Vpad): odd, >= nx + xp + kSepXB
__host__ __device__ constexpr int sep_bs(int nx, int px) { return (nx + sep_xp(px) + kSepXB) | 1; }

// the launch shape (index into kSepShapes) with the least FMA work per plane
// summed over the block's thread slots, tasks padded to whole lock-step
// groups (ties: the later shape, more tasks a thread); resident: every x task
// of the block fits at once (the forward keeps its x-pass outputs in
// registers across a depth chunk); -1 if none fits
inline int sep_pick_shape(int nx, int nz, int px, int pz, bool resident) {
  const int xtasks = nz * (nx / kSepXB), ztasks = nx * ((nz + kSepZB - 1) / kSepZB);
  int best = -1;
  double bc = 0;
  for (int i = 0; i < kSepNShapes; ++i) {
    const int nt = kSepShapes[i].nt, nth = kSepShapes[i].nth, nzt = (nt + 1) / 2;
    if (resident && nt * nth < xtasks) continue;
    const double xr = (xtasks + nt * nth - 1) / (nt * nth), zr = (ztasks + nzt * nth - 1) / (nzt * nth);
    const double c = (double)nth * (xr * nt * kSepXB * sep_xp(px) + zr * nzt * kSepZB * sep_zp(pz));
    if (best < 0 || c <= bc) {
      best = i;
      bc = c;
    }
  }
  return best;
}

struct SepArgs {
  int nx, ny, nz, px, pz;
  const float* P;        // forward input planes [nv][ny][nz][nx]
  float* T;              // adjoint output planes [nv][ny][nz][nx]
  const float* views;    // adjoint input views [nv][nz][nx]
  const float* att;      // attenuation cache [view][y][z][x]
  int att_mul;           // apply att (forward: on load, adjoint: on store)
  const float* H;        // [set][y][2 hs] weights (layout above)
  const float* tails;    // adjoint edge weights [set][y][ts] (see k_sconv_adj)
  int hs, ts;
  const int* vidx;       // [nv] plan view of each slot
  const int* viewset;    // [nview] PSF set of each view
  int nv, chunkY, nchunks;
  float* part;           // forward output [nv][nchunks][nz][nx]
  int* err;
};

// shared-memory bytes of k_sconv_fwd: staging (plane, attenuation, weights),
// mbarrier, working weights, ApadT [nx][rows | 1] (z fastest), Bz [nz][bs]
__host__ __device__ constexpr size_t sconv_fwd_smem(int nx, int nz, int px, int pz, int att) {
  return sizeof(float) * ((size_t)nx * nz * (att ? 2 : 1) + (sep_zp(pz) + sep_xp(px))) + 16 +
         sizeof(float) * (sep_zp(pz) + sep_xp(px)) + sizeof(float) * (size_t)(sep_rows(nz, pz) | 1) * nx +
         sizeof(float) * (size_t)nz * sep_bs(nx, px) + 16;
}

// one pass of NT tasks in lock step over contiguous padded lines: task i
// owns W consecutive outputs starting at base + off[i]:
// o[i][k] += sum_{m < len} w[m] base[off[i] + k + m]  (len a multiple of W,
// w 16-byte aligned); a sliding register window holds the W inputs in use
template <int NT, int W>
__device__ __forceinline__ void sep_pass(const float* __restrict__ w, int len, const float* base,
                                         const int (&off)[NT], float (&o)[NT][W]) {
  static_assert(W % 4 == 0, "window of whole float4 weight loads");
  float win[NT][W];
#pragma unroll
  for (int i = 0; i < NT; ++i)
#pragma unroll
    for (int j = 0; j < W; ++j) win[i][j] = base[off[i] + j];
  for (int m0 = 0; m0 < len; m0 += W) {
    float wv[W];
#pragma unroll
    for (int q = 0; q < W / 4; ++q) {
      const float4 w4 = *reinterpret_cast<const float4*>(w + m0 + 4 * q);
      wv[4 * q] = w4.x;
      wv[4 * q + 1] = w4.y;
      wv[4 * q + 2] = w4.z;
      wv[4 * q + 3] = w4.w;
    }
#pragma unroll
    for (int s = 0; s < W; ++s) {
#pragma unroll
      for (int i = 0; i < NT; ++i) {
#pragma unroll
        for (int k = 0; k < W; ++k) o[i][k] = fmaf(wv[s], win[i][(s + k) % W], o[i][k]);
        win[i][s] = base[off[i] + m0 + s + W];
      }
    }
  }
}

// k_sconv_fwd<NT, NTH>: persistent over items (slot, depth chunk) like
// k_conv_fwd2; NT = x-pass tasks per thread, NTH threads.  Per plane: the
// rotated plane,
// its attenuation plane and its weights are bulk-copied into shared memory
// one plane ahead (mbarrier, bounded wait); the block builds the attenuated,
// row-replicated plane Apad, runs the z pass into Bz (columns replicated),
// then the x pass, whose outputs stay in registers across the chunk; the
// chunk's partial view is written at its end.
template <int NT, int NTH>
__global__ void __launch_bounds__(NTH, 1) k_sconv_fwd(SepArgs a) {
  constexpr int NZ = (NT + 1) / 2;  // z-pass tasks per thread per group
  extern __shared__ float4 smem4[];
  const int nx = a.nx, nz = a.nz, px = a.px, pz = a.pz, hx = (px - 1) / 2, hz = (pz - 1) / 2;
  const int nplane = nx * nz, zp = sep_zp(pz), xp = sep_xp(px), hs = a.hs;
  const int bs = sep_bs(nx, px), rows = sep_rows(nz, pz), ast = rows | 1;
  // [sP][sA][sH][bar][Hw][ApadT][Bz]
  float* sP = reinterpret_cast<float*>(smem4);
  float* sA = sP + nplane;
  float* sH = sA + (a.att_mul ? nplane : 0);
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(sH + hs);
  float* Hw = reinterpret_cast<float*>(bar + 2);
  float* Apad = Hw + hs;  // transposed: column x at Apad + x * ast, row r = z + hz
  float* Bz = Apad + (size_t)ast * nx;
  const int nitems = a.nv * a.nchunks;
  const unsigned pbytes = (unsigned)(nplane * sizeof(float)), hbytes = (unsigned)(hs * sizeof(float));
  auto issue = [&](int item, int y) {  // one thread
    const int sl = item / a.nchunks, v = a.vidx[sl];
    fence_proxy_async();
    mbar_expect(bar, pbytes * (a.att_mul ? 2u : 1u) + hbytes);
    bulk_copy(bar, sP, a.P + ((size_t)sl * a.ny + y) * nplane, pbytes);
    if (a.att_mul) bulk_copy(bar, sA, a.att + ((size_t)v * a.ny + y) * nplane, pbytes);
    bulk_copy(bar, sH, a.H + ((size_t)a.viewset[v] * a.ny + y) * (2 * hs), hbytes);
  };
  if (threadIdx.x == 0) {
    mbar_init(bar);
    if ((int)blockIdx.x < nitems) issue(blockIdx.x, ((int)blockIdx.x % a.nchunks) * a.chunkY);
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const int nzb = (nz + kSepZB - 1) / kSepZB, ztasks = nx * nzb;
  const int xtasks = nz * (nx / kSepXB);
  // this thread's x tasks (z = t mod nz, x block = t / nz); tasks past the
  // end repeat the last one and are never stored
  int xoff[NT], xz[NT], xx[NT];
#pragma unroll
  for (int i = 0; i < NT; ++i) {
    const int t = min((int)threadIdx.x + i * NTH, xtasks - 1);
    const int xb = t / nz;
    xz[i] = t - xb * nz;
    xx[i] = xb * kSepXB;
    xoff[i] = xz[i] * bs + xx[i];
  }
  unsigned phase = 0;
  float acc[NT][kSepXB];
  for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
    const int slot = item / a.nchunks, ch = item - slot * a.nchunks;
    const int y0 = ch * a.chunkY, y1 = min(a.ny, y0 + a.chunkY);
#pragma unroll
    for (int i = 0; i < NT; ++i)
#pragma unroll
      for (int k = 0; k < kSepXB; ++k) acc[i][k] = 0.f;
    for (int y = y0; y < y1; ++y) {
      // staged plane y landed (the barrier also ends the previous x pass)
      if (__syncthreads_or(!mbar_wait(bar, phase))) {
        if (threadIdx.x == 0) {
          atomicExch(a.err, 1);
          mbar_wait(bar, phase);
        }
        return;
      }
      phase ^= 1u;
      // ApadT column x, entry r: plane row clamp(r - hz), attenuation applied
      for (int r = warp; r < rows; r += nwarps) {
        const int zs = min(max(r - hz, 0), nz - 1);
        const float* p = sP + zs * nx;
        const float* q = sA + zs * nx;
        for (int x = lane; x < nx; x += 32) Apad[x * ast + r] = a.att_mul ? __fmul_rn(p[x], q[x]) : p[x];
      }
      for (int k = threadIdx.x; k < hs; k += blockDim.x) Hw[k] = sH[k];
      __syncthreads();
      if (threadIdx.x == 0) {  // next plane of this block into the staging buffers
        if (y + 1 < y1) issue(item, y + 1);
        else if (item + (int)gridDim.x < nitems)
          issue(item + gridDim.x, ((item + (int)gridDim.x) % a.nchunks) * a.chunkY);
      }
      // z pass: tasks (x, z block), NZ per thread in lock step (groups of
      // NZ * blockDim tasks; tasks past the end repeat the last one, unstored)
      // -> Bz rows (columns c = x + hx, replicated at both ends)
      for (int tg = 0; tg < ztasks; tg += NZ * NTH) {
        int zoff[NZ], zz0[NZ], zx[NZ];
#pragma unroll
        for (int i = 0; i < NZ; ++i) {
          const int t = min(tg + (int)threadIdx.x + i * NTH, ztasks - 1);
          const int zb = t / nx;
          zx[i] = t - zb * nx;
          zz0[i] = zb * kSepZB;
          zoff[i] = zx[i] * ast + zz0[i];
        }
        float o[NZ][kSepZB];
#pragma unroll
        for (int i = 0; i < NZ; ++i)
#pragma unroll
          for (int k = 0; k < kSepZB; ++k) o[i][k] = 0.f;
        sep_pass<NZ, kSepZB>(Hw, zp, Apad, zoff, o);
#pragma unroll
        for (int i = 0; i < NZ; ++i) {
          const bool valid = tg + (int)threadIdx.x + i * NTH < ztasks;
          const int x = zx[i];
          if (valid)
#pragma unroll
            for (int k = 0; k < kSepZB; ++k)
              if (zz0[i] + k < nz) Bz[(size_t)(zz0[i] + k) * bs + x + hx] = o[i][k];
          // replicated edge columns (c < hx: column x = 0; c >= nx + hx:
          // x = nx - 1): the lane holding the edge task broadcasts its
          // outputs and the warp stores them (warp-uniform loop)
          unsigned m = __ballot_sync(0xffffffffu, valid && (x == 0 || x == nx - 1));
          while (m) {
            const int src = __ffs(m) - 1;
            m &= m - 1;
            const int sz0 = __shfl_sync(0xffffffffu, zz0[i], src), sx = __shfl_sync(0xffffffffu, x, src);
            const int c0 = sx == 0 ? 0 : nx + hx, c1 = sx == 0 ? hx : bs;
#pragma unroll
            for (int k = 0; k < kSepZB; ++k) {
              const float v = __shfl_sync(0xffffffffu, o[i][k], src);
              if (sz0 + k < nz)
                for (int c = c0 + lane; c < c1; c += 32) Bz[(size_t)(sz0 + k) * bs + c] = v;
            }
          }
        }
      }
      __syncthreads();
      // x pass, accumulated over the chunk
      sep_pass<NT, kSepXB>(Hw + zp, xp, Bz, xoff, acc);
    }
    // partial view of this chunk: part[slot][ch][z][x]
    float* out = a.part + ((size_t)slot * a.nchunks + ch) * nplane;
#pragma unroll
    for (int i = 0; i < NT; ++i)
      if ((int)threadIdx.x + i * NTH < xtasks)
#pragma unroll
        for (int q = 0; q < kSepXB / 4; ++q)
          *reinterpret_cast<float4*>(out + (size_t)xz[i] * nx + xx[i] + 4 * q) =
              make_float4(acc[i][4 * q], acc[i][4 * q + 1], acc[i][4 * q + 2], acc[i][4 * q + 3]);
  }
}

// shared-memory bytes of k_sconv_adj: two staging sets (attenuation plane,
// weights, edge tails), 2 mbarriers, Vpad [nz][bs], WpadT [nx][rows | 1]
__host__ __device__ constexpr size_t sconv_adj_smem(int nx, int nz, int px, int pz, int ts, int att) {
  return 2 * sizeof(float) * ((size_t)(att ? nx * nz : 0) + sep_zp(pz) + sep_xp(px) + ts) + 16 +
         sizeof(float) * (size_t)nz * sep_bs(nx, px) + sizeof(float) * (size_t)(sep_rows(nz, pz) | 1) * nx + 16;
}

// k_sconv_adj: the adjoint, fft_conv_adj! (src/fft_convolve.jl:82-130) for a
// factored plane: T = att .* Fz'(Fx'(V)).  The transpose of a clamped
// convolution F(v)[i] = sum_d a(d) v[clamp(i - d)] is the zero-padded
// correlation F'(u)[j] = sum_d a(d) u[j + d] plus, at the edges, the folded
// padding: F'(u)[0] += sum_{k<h} cL_k u[k], cL_k = sum_{d>k} a(d), and
// F'(u)[n-1] += sum_{k<h} cR_k u[n-1-k], cR_k = sum_{d<-k} a(d) (tails table
// [set][y][ts]: cL_x, cR_x, cL_z, cR_z, hx or hz values each).  Items (slot,
// depth chunk); the view is loaded zero-padded once per item; per plane the
// attenuation plane, weights and tails are bulk-copied two planes deep.
template <int NT, int NTH>
__global__ void __launch_bounds__(NTH, 1) k_sconv_adj(SepArgs a) {
  constexpr int NZ = (NT + 1) / 2;
  extern __shared__ float4 smem4[];
  const int nx = a.nx, nz = a.nz, px = a.px, pz = a.pz, hx = (px - 1) / 2, hz = (pz - 1) / 2;
  const int nplane = nx * nz, zp = sep_zp(pz), xp = sep_xp(px), hs = a.hs;
  const int bs = sep_bs(nx, px), rows = sep_rows(nz, pz), ast = rows | 1;
  const int sa = a.att_mul ? nplane : 0, stg = sa + hs + a.ts;
  // [stage 0: att, weights, tails][stage 1][bar x2][Vpad [nz][bs]][WpadT [nx][ast]]
  float* stage = reinterpret_cast<float*>(smem4);
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(stage + 2 * stg);
  float* Vpad = reinterpret_cast<float*>(bar + 2);
  float* Wpad = Vpad + (size_t)nz * bs;
  const int nitems = a.nv * a.nchunks;
  const unsigned pbytes = (unsigned)(nplane * sizeof(float));
  auto issue = [&](int item, int y, int b) {  // one thread
    const int sl = item / a.nchunks, v = a.vidx[sl], set = a.viewset[v];
    float* st = stage + b * stg;
    fence_proxy_async();
    mbar_expect(&bar[b], (a.att_mul ? pbytes : 0u) + (unsigned)((hs + a.ts) * sizeof(float)));
    if (a.att_mul) bulk_copy(&bar[b], st, a.att + ((size_t)v * a.ny + y) * nplane, pbytes);
    bulk_copy(&bar[b], st + sa, a.H + ((size_t)set * a.ny + y) * (2 * hs) + hs, (unsigned)(hs * sizeof(float)));
    bulk_copy(&bar[b], st + sa + hs, a.tails + ((size_t)set * a.ny + y) * a.ts, (unsigned)(a.ts * sizeof(float)));
  };
  // the sequence of (item, plane) of this block
  auto next = [&](int& item, int& y) {
    const int y1 = min(a.ny, (item % a.nchunks) * a.chunkY + a.chunkY);
    if (y + 1 < y1) {
      ++y;
    } else {
      item += gridDim.x;
      y = (item % a.nchunks) * a.chunkY;
    }
  };
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  // WpadT entries outside the image rows (r < hz, r >= hz + nz) stay zero
  for (int x = warp; x < nx; x += nwarps)
    for (int r = lane; r < ast; r += 32)
      if (r < hz || r >= hz + nz) Wpad[(size_t)x * ast + r] = 0.f;
  // planes in consumption order P0, P1, ...: P0 -> stage 0, P1 -> stage 1;
  // every thread tracks the queue head (the next plane to issue)
  int qi = blockIdx.x, qy = (blockIdx.x % a.nchunks) * a.chunkY;  // P0
  int i1 = qi, y1q = qy;
  next(i1, y1q);  // P1
  if (threadIdx.x == 0) {
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
  next(qi, qy);  // P2
  if (!((int)blockIdx.x < nitems)) return;
  const int nzb = (nz + kSepZB - 1) / kSepZB, ztasks = nx * nzb;
  const int xtasks = nz * (nx / kSepXB);
  unsigned phases = 0u;
  int b = 0;
  for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
    const int slot = item / a.nchunks, ch = item - slot * a.nchunks;
    const int y0 = ch * a.chunkY, y1 = min(a.ny, y0 + a.chunkY);
    // the view, zero-padded: Vpad[z][c] = V[z][c - hx] (previous item's
    // passes are done: the barrier at the end of each plane)
    const float* V = a.views + (size_t)slot * nplane;
    for (int z = warp; z < nz; z += nwarps) {
      float* row = Vpad + (size_t)z * bs;
      for (int c = lane; c < bs; c += 32) row[c] = (c >= hx && c < hx + nx) ? V[z * nx + c - hx] : 0.f;
    }
    for (int y = y0; y < y1; ++y) {
      const unsigned par = (phases >> b) & 1u;
      if (__syncthreads_or(!mbar_wait(&bar[b], par))) {
        if (threadIdx.x == 0) {
          atomicExch(a.err, 1);
          mbar_wait(&bar[b], par);
        }
        return;
      }
      phases ^= 1u << b;
      const float* st = stage + b * stg;
      const float* sA = st;
      const float* bz = st + sa;         // b[m], zero-padded to zp
      const float* ax = bz + zp;         // a[m], zero-padded to xp
      const float* tl = st + sa + hs;    // cL_x, cR_x, cL_z, cR_z
      // x pass: Fx' of the view -> Wpad rows hz .. hz + nz - 1 (NT tasks per
      // thread in lock step, in groups of NT * blockDim)
      for (int tg = 0; tg < xtasks; tg += NT * NTH) {
        int off[NT], xz[NT], x0s[NT];
#pragma unroll
        for (int i = 0; i < NT; ++i) {
          const int t = min(tg + (int)threadIdx.x + i * NTH, xtasks - 1);
          const int xb = t / nz;
          xz[i] = t - xb * nz;
          x0s[i] = xb * kSepXB;
          off[i] = xz[i] * bs + x0s[i];
        }
        float o[NT][kSepXB];
#pragma unroll
        for (int i = 0; i < NT; ++i)
#pragma unroll
          for (int k = 0; k < kSepXB; ++k) o[i][k] = 0.f;
        sep_pass<NT, kSepXB>(ax, xp, Vpad, off, o);
#pragma unroll
        for (int i = 0; i < NT; ++i) {
          if (tg + (int)threadIdx.x + i * NTH >= xtasks) continue;
          const int x0 = x0s[i];
          const float* row = Vpad + off[i];
          if (x0 == 0)
            for (int k = 0; k < hx; ++k) o[i][0] = fmaf(tl[k], row[hx + k], o[i][0]);
          if (x0 + kSepXB == nx)
            for (int k = 0; k < hx; ++k)
              o[i][kSepXB - 1] = fmaf(tl[hx + k], row[hx + kSepXB - 1 - k], o[i][kSepXB - 1]);
          float* w = Wpad + (size_t)x0 * ast + xz[i] + hz;
#pragma unroll
          for (int k = 0; k < kSepXB; ++k) w[(size_t)k * ast] = o[i][k];
        }
      }
      __syncthreads();
      // z pass: Fz' -> T plane, times the attenuation (NZ tasks per thread)
      float* Tp = a.T + ((size_t)slot * a.ny + y) * nplane;
      for (int tg = 0; tg < ztasks; tg += NZ * NTH) {
        int zoff[NZ], zz0[NZ], zx[NZ];
#pragma unroll
        for (int i = 0; i < NZ; ++i) {
          const int t = min(tg + (int)threadIdx.x + i * NTH, ztasks - 1);
          const int zb = t / nx;
          zx[i] = t - zb * nx;
          zz0[i] = zb * kSepZB;
          zoff[i] = zx[i] * ast + zz0[i];
        }
        float o[NZ][kSepZB];
#pragma unroll
        for (int i = 0; i < NZ; ++i)
#pragma unroll
          for (int k = 0; k < kSepZB; ++k) o[i][k] = 0.f;
        sep_pass<NZ, kSepZB>(bz, zp, Wpad, zoff, o);
#pragma unroll
        for (int i = 0; i < NZ; ++i) {
          if (tg + (int)threadIdx.x + i * NTH >= ztasks) continue;
          const int z0 = zz0[i], x = zx[i];
          const float* img = Wpad + (size_t)x * ast + hz;  // Fx'(V) row z at img[z]
          if (z0 == 0)
            for (int k = 0; k < hz; ++k) o[i][0] = fmaf(tl[2 * hx + k], img[k], o[i][0]);
#pragma unroll
          for (int k = 0; k < kSepZB; ++k) {
            const int z = z0 + k;
            if (z == nz - 1)
              for (int q = 0; q < hz; ++q) o[i][k] = fmaf(tl[2 * hx + hz + q], img[nz - 1 - q], o[i][k]);
            if (z < nz) Tp[(size_t)z * nx + x] = a.att_mul ? __fmul_rn(sA[z * nx + x], o[i][k]) : o[i][k];
          }
        }
      }
      __syncthreads();
      if (threadIdx.x == 0 && qi < nitems) issue(qi, qy, b);  // this stage set is free again
      next(qi, qy);
      b ^= 1;
    }
  }
}

}  // namespace spect
