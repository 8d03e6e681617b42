// zpath_inst.cu -- instantiations and launchers of the fused projector pair
// (zpath.cuh), compiled as a unit of its own.
#include "zpath.cuh"

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

template <int ZPL>
cudaError_t zrot(const ZGeom& g, int grid, cudaStream_t st, const float* T, const float4* rot, const int* vidx,
                 int nv, const float* prev, float* out, const float* x, const float* asum, int mode) {
  k_zrot_adj<ZPL><<<grid, 256, 0, st>>>(g, T, rot, vidx, nv, prev, out, x, asum, mode);
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
