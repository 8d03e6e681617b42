// conv_inst.cu -- instantiates the convolution kernels of conv2.cuh for one
// value of RX (compiled once per RX in {1,2,4,8,16} with -DSPECT_RX=RX) and
// all RZ; spect_gpu.cu dispatches on (RX, RZ).
#include "conv2.cuh"

#ifndef SPECT_RX
#error "compile with -DSPECT_RX=<1|2|4|8|16>"
#endif

#define SPECT_CAT2(a, b) a##b
#define SPECT_CAT(a, b) SPECT_CAT2(a, b)

namespace spect {

namespace {
// kind 0 forward, 1 adjoint, 2 view spectra, 3 forward with plane staging,
// 4 adjoint with staged attenuation multiplied on store
template <int RZ>
const void* kernel_ptr(int kind) {
  constexpr bool REG = SPECT_RX * RZ <= 32;
  if (kind == 0) return (const void*)k_conv_fwd2<SPECT_RX, RZ, REG, false>;
  if (kind == 3) return (const void*)k_conv_fwd2<SPECT_RX, RZ, REG, true>;
  if (kind == 1) return (const void*)k_conv_adj2<SPECT_RX, RZ, REG, false>;
  if (kind == 4) return (const void*)k_conv_adj2<SPECT_RX, RZ, REG, true>;
  return (const void*)k_vspec2<SPECT_RX, RZ>;
}
const void* kernel_ptr_rt(int kind, int RZ) {
  switch (RZ) {
    case 1: return kernel_ptr<1>(kind);
    case 2: return kernel_ptr<2>(kind);
    case 4: return kernel_ptr<4>(kind);
    case 8: return kernel_ptr<8>(kind);
    case 16: return kernel_ptr<16>(kind);
  }
  return nullptr;
}
}  // namespace

cudaError_t SPECT_CAT(conv2_launch_rx, SPECT_RX)(int kind, int RZ, int grid, size_t smem, cudaStream_t st,
                                                 const Conv2Args& a) {
  const void* k = kernel_ptr_rt(kind, RZ);
  if (!k) return cudaErrorInvalidValue;
  Conv2Args arg = a;
  void* params[] = {&arg};
  return cudaLaunchKernel(k, dim3(grid), dim3(kConvThreads), params, smem, st);
}

// The attribute is set to the device's opt-in maximum (plans of different
// sizes share the instantiation; each launch passes its own size).
cudaError_t SPECT_CAT(conv2_setup_rx, SPECT_RX)(int RZ, size_t smem, int* occ) {
  int o = 64, dev = 0, optin = 0;
  cudaError_t e0 = cudaGetDevice(&dev);
  if (e0 == cudaSuccess) e0 = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e0 != cudaSuccess) return e0;
  for (int kind = 0; kind < 5; ++kind) {
    const void* k = kernel_ptr_rt(kind, RZ);
    if (!k) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    if (e != cudaSuccess) return e;
    int b = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k, kConvThreads, smem);
    if (e != cudaSuccess) return e;
    o = b < o ? b : o;
  }
  *occ = o;
  return cudaSuccess;
}

}  // namespace spect
