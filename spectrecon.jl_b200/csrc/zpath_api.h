// zpath_api.h -- host-visible part of the fused projector pair (zpath.cuh):
// geometry of the z-fastest layouts, kernel arguments, shared-memory sizes and
// the launchers defined in zpath_inst.cu.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

namespace spect {

// sizes shared by the zpath kernels (computed once per plan on the host)
struct ZGeom {
  int nx, ny, nz, nzp, L, pad;
  float c0;         // rotation centre (nx - 1)/2, 0-based
  int px, pz, hx, hz;
  int R0, C0;       // first data row (z pass) / column (x pass) of the padded buffers
  int zpw, xpw;     // window taps of the z and x passes (shifted, multiples of 8)
  int hs, ts;       // weight-row and tail-row lengths of one direction
  int rows, ast;    // z-pass buffer: rows per column, column stride (4 * odd)
  int bs;           // x-pass buffer row stride (4 * odd)
  int nwa;          // k_zadj x-pass output buffers: 2 (double-buffered) or 1
  int nsf;          // k_zfwd staging buffers: 2 (two planes in flight) or 1
};

__host__ __device__ constexpr int zround(int v, int m) { return (v + m - 1) / m * m; }
// smallest 4 * odd >= v: 16-byte rows whose float4 chunk index is odd, so the
// eight lanes of a 128-bit shared access phase hit distinct bank groups
__host__ __device__ constexpr int zstride4(int v) {
  return ((zround(v, 4) / 4) % 2 == 1) ? zround(v, 4) : zround(v, 4) + 4;
}

inline ZGeom zgeom_make(int nx, int ny, int nz, int px, int pz, int pad) {
  ZGeom g{};
  g.nx = nx;
  g.ny = ny;
  g.nz = nz;
  g.nzp = zround(nz, 16);
  g.pad = pad;
  g.L = nx + 2 * pad;
  g.c0 = (float)((nx - 1) * 0.5);
  g.px = px;
  g.pz = pz;
  g.hx = (px - 1) / 2;
  g.hz = (pz - 1) / 2;
  g.R0 = zround(g.hz, 4);
  g.C0 = zround(g.hx, 4);
  g.zpw = zround(g.R0 - g.hz + pz, 8);
  g.xpw = zround(g.C0 - g.hx + px, 8);
  g.hs = g.zpw + g.xpw;
  g.ts = zround(2 * g.hx + 2 * g.hz, 4) < 4 ? 4 : zround(2 * g.hx + 2 * g.hz, 4);
  g.rows = zround(nz, 16) + g.zpw;  // z tasks of 8 or 16 outputs
  g.ast = zstride4(g.rows);
  g.bs = zstride4(nx + g.xpw);
  g.nwa = 1;
  g.nsf = 1;
  return g;
}

struct ZArgs {
  ZGeom g;
  const float* img;     // IZ
  const float* att;     // ATT
  const float* H;       // [set][y][2 hs]: fwd z | fwd x | adj z | adj x
  const float* E;       // [set][y][2 ts]: ELz ERz ELx ERx | cLx cRx cLz cRz
  const int* R;         // [set][y][8]: (first 4-tap block, 8-tap blocks) of fwd z | fwd x | adj z | adj x
  const float4* rot;    // [view] (cos(2pi - theta), sin(2pi - theta), theta == 0, theta)
  const int* vidx;      // [nv] plan view of each slot
  const int* viewset;   // [nview] PSF set of each view
  int nv, chunkY, nchunks;
  float* part;          // k_zfwd output [nv][nchunks][nz][nx]
  const float* views;   // k_zadj input [nv][nz][nx]
  float* T;             // k_zadj output [nv][ny][nx][nzp]
  int* err;
  float* Q;             // plane-tile exchange of the large-plane kernels (zstrip.cuh)
  int tx, tz;           // their column and row tile sizes
};

// k_zfwd shared memory (floats; every region 16-byte aligned):
//   [bar 4][nsf stages: att plane nx*nzp | weights hs | tails ts | ranges 4]
//   [Hw 2 x (hs + ts + 4)][geoW nx (float4)][geoO nx (int), rounded to 4]
//   [ZB nx * ast][XB nz * bs]
__host__ __device__ inline size_t zfwd_smem(const ZGeom& g, int nsf) {
  const size_t f = 4 + nsf * ((size_t)g.nx * g.nzp + g.hs + g.ts + 4) + 2 * (size_t)(g.hs + g.ts + 4) +
                   4 * (size_t)g.nx + zround(g.nx, 4) + (size_t)g.nx * g.ast + (size_t)g.nz * g.bs;
  return f * sizeof(float);
}

// k_zadj shared memory (floats): [bar 8][3 stages x (weights hs | folds ts | ranges 4)]
//   [VB nz * bs: the view, zero-padded, data columns C0..][nwb x WB nx * ast:
//   x-pass output, column x, data rows R0..]
__host__ __device__ inline size_t zadj_smem(const ZGeom& g, int nwb) {
  return sizeof(float) *
         (8 + 3 * (size_t)(g.hs + g.ts + 4) + (size_t)g.nz * g.bs + (size_t)nwb * g.nx * g.ast);
}

// launch shapes of k_zfwd / k_zadj: NT tasks of W outputs per thread, NTH
// threads (W = 16 needs nx % 16 == 0); fwd: the forward compiles without
// register spills in this shape (with the accumulators, 1024 threads and the
// largest NT leave too few registers)
struct ZShape {
  int nt, nth, w, fwd;
};
constexpr int kZNShapes = 13;
constexpr ZShape kZShapes[kZNShapes] = {{1, 512, 8, 1},  {2, 512, 8, 1},  {3, 512, 8, 1},   {4, 512, 8, 0},
                                        {1, 640, 8, 1},  {2, 640, 8, 1},  {3, 640, 8, 0},   {1, 1024, 8, 0},
                                        {1, 512, 16, 1}, {2, 512, 16, 1}, {1, 640, 16, 1},  {2, 640, 16, 0},
                                        {1, 1024, 16, 0}};
inline bool zfwd_shape_ok(int i) { return kZShapes[i].fwd != 0; }
inline bool zshape_fits(const ZGeom& g, int i) { return g.nx % kZShapes[i].w == 0; }

// large-plane kernels (zstrip.cuh), shared memory in bytes
__host__ __device__ inline size_t zs_fz_smem(const ZGeom& g, int tx) {
  return sizeof(float) * ((size_t)g.hs + g.ts + 4 + 5 * (size_t)tx + (size_t)tx * g.ast + (size_t)g.nz * tx);
}
__host__ __device__ inline size_t zs_fx_smem(const ZGeom& g, int tz) {
  return sizeof(float) * 2 * ((size_t)tz * g.bs + g.hs + g.ts + 4);
}
__host__ __device__ inline size_t zs_adj_smem(const ZGeom& g, int tx) {
  return sizeof(float) * ((size_t)g.nz * zstride4(tx + g.xpw) + (size_t)tx * g.ast + g.hs + g.ts + 4);
}
struct ZsTiles {
  int w, tx, tz;  // task width, column tile, row tile
};
constexpr int kZsNth = 512;   // k_zs_fz, k_zs_adj threads
constexpr int kZsNthX = 640;  // k_zs_fx threads (one x task each)

// launchers (zpath_inst.cu)
cudaError_t zpath_setup(int max_smem);
cudaError_t zfwd_launch(int shape, int grid, size_t smem, cudaStream_t st, const ZArgs& a);
cudaError_t zadj_launch(int shape, int grid, size_t smem, cudaStream_t st, const ZArgs& a);
cudaError_t zrot_adj_launch(const ZGeom& g, int grid, cudaStream_t st, const float* T, const float4* rot,
                            const int* vidx, int nv, const float* prev, float* out, const float* x, const float* asum,
                            int mode);
cudaError_t zto_iz_launch(const ZGeom& g, cudaStream_t st, const float* img, float* iz);
cudaError_t zt_to_z_launch(const ZGeom& g, int planes, cudaStream_t st, const float* src, float* dst,
                            const float* att, const int* vidx);
cudaError_t zfrom_iz_launch(const ZGeom& g, cudaStream_t st, const float* iz, float* dst, const float* asum, int mode);
// large-plane kernels: w = task width (8 or 16); occ = resident blocks per
// SM of k_zs_fz, k_zs_fx, k_zs_adj at their shared-memory sizes (for the
// persistent grids)
cudaError_t zstrip_setup(int max_smem);
cudaError_t zstrip_occupancy(int w, int fz_nth, int adj_nth, const size_t smem[3], int occ[3]);
cudaError_t zs_fz_launch(int w, int nth, int grid, size_t smem, cudaStream_t st, const ZArgs& a);
cudaError_t zs_fx_launch(int w, int grid, size_t smem, cudaStream_t st, const ZArgs& a);
cudaError_t zs_adj_launch(int w, int nth, int grid, size_t smem, cudaStream_t st, const ZArgs& a);
cudaError_t zatten_launch(const ZGeom& g, int nview, cudaStream_t st, const float* muz, const float4* rot, float dy,
                          float* att);

}  // namespace spect
