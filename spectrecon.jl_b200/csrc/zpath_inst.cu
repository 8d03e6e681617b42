// zpath_inst.cu -- instantiations and launchers of the fused projector pair
// (zpath.cuh) and of the large-plane kernels (zstrip.cuh), compiled as a unit
// of its own.
#include <cstdlib>

#include "zpath.cuh"
#include "zstrip.cuh"

namespace spect {

namespace {
// the order of kZShapes
#define ZSHAPES(K)                                                                                           \
  {(const void*)K<1, 512, 8>,  (const void*)K<2, 512, 8>,   (const void*)K<3, 512, 8>,                       \
   (const void*)K<4, 512, 8>,  (const void*)K<1, 640, 8>,   (const void*)K<2, 640, 8>,                       \
   (const void*)K<3, 640, 8>,  (const void*)K<1, 1024, 8>,  (const void*)K<1, 512, 16>,                      \
   (const void*)K<2, 512, 16>, (const void*)K<1, 640, 16>,  (const void*)K<2, 640, 16>,                      \
   (const void*)K<1, 1024, 16>}
const void* const kZfwd[kZNShapes] = ZSHAPES(k_zfwd);
const void* const kZadj[kZNShapes] = ZSHAPES(k_zadj);
#undef ZSHAPES

// k_zrot_adj's candidates per load round: the largest of 3 and 2 whose
// rounds compile without register spills under the kernel's launch bounds
// (64 registers per thread for ZPL <= 14, 128 above; from ptxas -v for
// every ZPL); 0 (one branch per candidate) where both spill.
// SPECT_ZROT_RB=0 selects the branch form everywhere; read once per process.
constexpr int zrot_rounds(int zpl) {
  return (zpl <= 10 || (zpl >= 16 && zpl <= 24)) ? 3 : (zpl == 26 || zpl >= 30) ? 2 : 0;
}
bool zrot_branch_form() {
  static const bool b = [] {
    const char* e = getenv("SPECT_ZROT_RB");
    return e != nullptr && e[0] == '0' && e[1] == 0;
  }();
  return b;
}

template <int ZPL>
cudaError_t zrot(const ZGeom& g, int grid, cudaStream_t st, const float* T, const float4* rot, const int* vidx,
                 int nv, const float* prev, float* out, const float* x, const float* asum, int mode) {
  if (zrot_branch_form())
    k_zrot_adj<ZPL, 0><<<grid, 256, 0, st>>>(g, T, rot, vidx, nv, prev, out, x, asum, mode);
  else
    k_zrot_adj<ZPL, zrot_rounds(ZPL)><<<grid, 256, 0, st>>>(g, T, rot, vidx, nv, prev, out, x, asum, mode);
  return cudaGetLastError();
}
}  // namespace

cudaError_t zpath_setup(int max_smem) {
  for (int i = 0; i < kZNShapes; ++i) {
    cudaError_t e = cudaFuncSetAttribute(kZfwd[i], cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(kZadj[i], cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t zfwd_launch(int shape, int grid, size_t smem, cudaStream_t st, const ZArgs& a) {
  ZArgs c = a;
  void* args[] = {&c};
  return cudaLaunchKernel(kZfwd[shape], dim3(grid), dim3(kZShapes[shape].nth), args, smem, st);
}

cudaError_t zadj_launch(int shape, int grid, size_t smem, cudaStream_t st, const ZArgs& a) {
  ZArgs c = a;
  void* args[] = {&c};
  return cudaLaunchKernel(kZadj[shape], dim3(grid), dim3(kZShapes[shape].nth), args, smem, st);
}

cudaError_t zrot_adj_launch(const ZGeom& g, int grid, cudaStream_t st, const float* T, const float4* rot,
                            const int* vidx, int nv, const float* prev, float* out, const float* x, const float* asum,
                            int mode) {
  switch (g.nzp / 8) {  // nzp is a multiple of 16
#define ZCASE(n) \
  case n: return zrot<n>(g, grid, st, T, rot, vidx, nv, prev, out, x, asum, mode);
    ZCASE(2) ZCASE(4) ZCASE(6) ZCASE(8) ZCASE(10) ZCASE(12) ZCASE(14) ZCASE(16)
    ZCASE(18) ZCASE(20) ZCASE(22) ZCASE(24) ZCASE(26) ZCASE(28) ZCASE(30) ZCASE(32)
#undef ZCASE
  }
  return cudaErrorInvalidValue;
}

namespace {
// k_zs_fz: 512 threads (index 0, 1) or 256 (index 2, 3: two blocks per SM at these registers)
const void* const kZsFz[4] = {(const void*)k_zs_fz<kZsNth, 8>, (const void*)k_zs_fz<kZsNth, 16>,
                              (const void*)k_zs_fz<kZsNth / 2, 8>, (const void*)k_zs_fz<kZsNth / 2, 16>};
const void* const kZsFx[2] = {(const void*)k_zs_fx<kZsNthX, 8>, (const void*)k_zs_fx<kZsNthX, 16>};
// k_zs_adj: 512 threads (index 0, 1) or 256 (index 2, 3: narrower tiles, two blocks per SM)
const void* const kZsAdj[4] = {(const void*)k_zs_adj<kZsNth, 8>, (const void*)k_zs_adj<kZsNth, 16>,
                               (const void*)k_zs_adj<kZsNth / 2, 8>, (const void*)k_zs_adj<kZsNth / 2, 16>};
cudaError_t zs_launch(const void* k, int nth, int grid, size_t smem, cudaStream_t st, const ZArgs& a) {
  ZArgs c = a;
  void* args[] = {&c};
  return cudaLaunchKernel(k, dim3(grid), dim3(nth), args, smem, st);
}
}  // namespace

cudaError_t zstrip_setup(int max_smem) {
  for (int i = 0; i < 2; ++i)
    for (const void* k : {kZsFz[i], kZsFz[i + 2], kZsFx[i], kZsAdj[i], kZsAdj[i + 2]}) {
      const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem);
      if (e != cudaSuccess) return e;
    }
  return cudaSuccess;
}

cudaError_t zstrip_occupancy(int w, int fz_nth, int adj_nth, const size_t smem[3], int occ[3]) {
  const int i = w == 16 ? 1 : 0, f = fz_nth == kZsNth ? i : i + 2, d = adj_nth == kZsNth ? i : i + 2;
  const void* ks[3] = {kZsFz[f], kZsFx[i], kZsAdj[d]};
  const int nth[3] = {fz_nth, kZsNthX, adj_nth};
  for (int j = 0; j < 3; ++j) {
    const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[j], ks[j], nth[j], smem[j]);
    if (e != cudaSuccess) return e;
    if (occ[j] < 1) occ[j] = 1;
  }
  return cudaSuccess;
}

cudaError_t zs_fz_launch(int w, int nth, int grid, size_t smem, cudaStream_t st, const ZArgs& a) {
  return zs_launch(kZsFz[(w == 16 ? 1 : 0) + (nth == kZsNth ? 0 : 2)], nth, grid, smem, st, a);
}
cudaError_t zs_fx_launch(int w, int grid, size_t smem, cudaStream_t st, const ZArgs& a) {
  return zs_launch(kZsFx[w == 16 ? 1 : 0], kZsNthX, grid, smem, st, a);
}
cudaError_t zs_adj_launch(int w, int nth, int grid, size_t smem, cudaStream_t st, const ZArgs& a) {
  return zs_launch(kZsAdj[(w == 16 ? 1 : 0) + (nth == kZsNth ? 0 : 2)], nth, grid, smem, st, a);
}

cudaError_t zto_iz_launch(const ZGeom& g, cudaStream_t st, const float* img, float* iz) {
  k_to_iz<<<dim3((g.nx + 31) / 32, g.ny, (g.nzp + 31) / 32), dim3(32, 8), 0, st>>>(g, img, iz);
  return cudaGetLastError();
}

cudaError_t zt_to_z_launch(const ZGeom& g, int planes, cudaStream_t st, const float* src, float* dst,
                            const float* att, const int* vidx) {
  k_t_to_z<<<dim3((g.nx + 31) / 32, planes, (g.nzp + 31) / 32), dim3(32, 8), 0, st>>>(g, src, dst, att, vidx);
  return cudaGetLastError();
}

cudaError_t zfrom_iz_launch(const ZGeom& g, cudaStream_t st, const float* iz, float* dst, const float* asum, int mode) {
  k_from_iz<<<dim3((g.nx + 31) / 32, g.ny, (g.nz + 31) / 32), dim3(32, 8), 0, st>>>(g, iz, dst, asum, mode);
  return cudaGetLastError();
}

cudaError_t zatten_launch(const ZGeom& g, int nview, cudaStream_t st, const float* muz, const float4* rot, float dy,
                          float* att) {
  k_zatten<<<dim3(g.nx, nview), g.nzp, 0, st>>>(g, muz, rot, dy, att);
  return cudaGetLastError();
}

}  // namespace spect
