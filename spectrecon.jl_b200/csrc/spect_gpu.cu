// spect_gpu.cu -- C ABI of the B200 SPECT projector (declared in include/spect_gpu.h).
//
// Host side of the drop-in boundary: SPECTplan construction and validation
// (src/spectplan.jl:58-137), project!/backproject! over a view index list
// (src/project.jl:143-163, src/backproject.jl:132-162), ML-EM / OS-EM with the
// EM ratio and multiplicative update fused into the projector's last stages
// (src/ml-os-em.jl:21-131), and psf_gauss (src/psf-gauss.jl:24-55).
//
// Device memory layout (HBM), all float32 unless noted:
//   mumap   [nz][ny][nx]                 uploaded once per plan
//   Hs      [nset][ny][Q+1][Npx]         real PSF spectra / (Npx*Npz) in the
//                                        scrambled orders of conv2.cuh, one set
//                                        per distinct psfs[:,:,:,v] (views with
//                                        identical PSF stacks share a set)
//   P / T   [gmax][ny][nz][nx]           rotated+attenuated planes (forward) /
//                                        adjoint-convolved planes (adjoint) of
//                                        one group of views
//   part    [gmax][nchunk][nz][nx]       per depth-chunk partial views
//   Vs      [gmax][Q][Npx] complex       spectra of the views (adjoint)
//   imgpart [nsplit][nz][ny][nx]         per view-split partial images
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/spect_gpu.h"
#include "conv2.cuh"
#include "rot_one.cuh"
#include "sconv.cuh"
#include "spect_kernels.cuh"
#include "zpath_api.h"

using namespace spect;

namespace spect {
// per-RX instantiation units (conv_inst.cu)
#define SPECT_DECL_RX(n)                                                                                   \
  cudaError_t conv2_launch_rx##n(int kind, int RZ, int grid, size_t smem, cudaStream_t st, const Conv2Args& a); \
  cudaError_t conv2_setup_rx##n(int RZ, size_t smem, int* occ);
SPECT_DECL_RX(1)
SPECT_DECL_RX(2)
SPECT_DECL_RX(4)
SPECT_DECL_RX(8)
SPECT_DECL_RX(16)
#undef SPECT_DECL_RX
}  // namespace spect

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CUDA_TRY(expr)                                                                                  \
  do {                                                                                                  \
    cudaError_t e_ = (expr);                                                                            \
    if (e_ != cudaSuccess) {                                                                            \
      return fail(e_ == cudaErrorMemoryAllocation ? SPECT_ERR_OOM : SPECT_ERR_CUDA,                     \
                  std::string(#expr) + ": " + cudaGetErrorString(e_));                                  \
    }                                                                                                   \
  } while (0)

#define STATUS_TRY(expr)       \
  do {                         \
    int st_ = (expr);          \
    if (st_ != SPECT_OK) return st_; \
  } while (0)

inline int power2(int x) {
  int p = 1;
  while (p < x) p <<= 1;
  return p;
}
inline int ilog2(int x) {
  int l = 0;
  while ((1 << l) < x) ++l;
  return l;
}
inline int cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }

constexpr double kTwoPi = 6.283185307179586;

std::atomic<unsigned long long> g_launches{0};

enum KernelKind { K_ROT_FWD, K_CONV_FWD, K_REDUCE_VIEWS, K_VSPEC, K_CONV_ADJ, K_ROT_ADJ, K_REDUCE_IMAGE, K_OTHER,
                  K_KINDS };

// CUDA-event bracketing of every launch of a plan (measurement support)
struct Profiler {
  bool on = false;
  struct Rec {
    int kind;
    cudaEvent_t a, b;
  };
  std::vector<Rec> pending;
  std::vector<cudaEvent_t> pool;
  double ms[K_KINDS] = {0};
  long long n[K_KINDS] = {0};
  cudaEvent_t get() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
  void drain() {
    for (auto& r : pending) {
      cudaEventSynchronize(r.b);
      float t = 0;
      cudaEventElapsedTime(&t, r.a, r.b);
      ms[r.kind] += t;
      n[r.kind] += 1;
      pool.push_back(r.a);
      pool.push_back(r.b);
    }
    pending.clear();
  }
  void reset() {
    drain();
    for (int k = 0; k < K_KINDS; ++k) {
      ms[k] = 0;
      n[k] = 0;
    }
  }
  ~Profiler() {
    for (auto& r : pending) {
      cudaEventDestroy(r.a);
      cudaEventDestroy(r.b);
    }
    for (auto e : pool) cudaEventDestroy(e);
  }
};

}  // namespace

struct spect_plan_s {
  int nx, ny, nz, px, pz, nview, interp, mode, nthread;
  float dy;
  Geom g;
  int device = 0, sm_count = 148;
  size_t max_smem = 232448;
  int nset = 0;
  std::vector<int> view_set;
  std::vector<float> angles;
  size_t N = 0, nxz = 0;
  // device
  float* d_mumap = nullptr;
  float* d_att = nullptr;  // [nview][ny][nz][nx] attenuation cache (optional for :two, required for :one)
  // :one rotation
  Rot1Geom r1;
  Rot1View* d_r1view = nullptr;
  float* d_R1 = nullptr;       // [gmax][nz][ny][nx] rotated slices / attenuated adjoint planes
  float* d_gscr_r1 = nullptr;  // per-CTA work grids when they do not fit in shared memory
  size_t r1f_smem = 0, r1a_smem = 0;
  int r1f_smem_ok = 1, r1a_smem_ok = 1, r1_grid_y = 1;
  float* d_H = nullptr;
  float4* d_rot = nullptr;
  int* d_viewset = nullptr;
  float2* d_tw = nullptr;
  int* d_all = nullptr;  // 0..nview-1
  int* d_idx = nullptr;  // per-call index staging [nview]
  // work scratch for one group of views
  int gmax = 1, nchunk_max = 32;
  float* d_P = nullptr;
  float* d_part = nullptr;
  float2* d_Vs = nullptr;
  float* d_imgpart = nullptr;
  float2* d_gB = nullptr;
  float2* d_gacc = nullptr;
  // separable PSF planes: direct-FMA convolution (sconv.cuh)
  // sep_fwd_ok / sep_adj_ok: the direct kernels can run; sep / sep_adj: they
  // are in use (default on; the autotuner keeps the faster of direct and FFT)
  int sep_ok = 0, sep = 0, sep_adj = 0, sep_hs = 0, sep_ts = 0;
  int sep_shape_fwd = -1, sep_shape_adj = -1;  // indices into kSepShapes
  int sep_fwd_ok = 0, sep_adj_ok = 0, sep_forced = 0;  // forced: 1 FFT, 2 direct
  float* d_Hsep = nullptr;      // [nset][ny][sep_hs] reversed z, x factors
  float* d_Tsep = nullptr;      // [nset][ny][sep_ts] adjoint edge tails
  size_t sep_fwd_smem = 0, sep_adj_smem = 0;
  float* d_gscr_adj = nullptr;
  // EM scratch (lazily allocated)
  float* d_views_tmp = nullptr;  // [nview][nz][nx]
  float* d_ones = nullptr;       // [nview][nz][nx]
  float* d_asum = nullptr;       // [nblocks][N]
  int asum_blocks = 0;
  int* d_sub = nullptr;          // [nview] subset view table of the last prepared nblocks
  int sub_nblocks = 0;
  int* d_flag = nullptr;
  // host-call staging (lazily allocated)
  float* d_io_img = nullptr;   // [2][N]
  float* d_io_views = nullptr; // [3][nview][nz][nx]
  // launch configuration
  ConvGeom cg;
  int RX = 1, RZ = 1;
  int conv_grid = 148, conv_bsmem = 1;
  size_t conv_smem = 0;
  int conv_stage = 0;         // forward kernel stages planes by bulk copy
  size_t conv_smem_fwd = 0;   // its shared memory
  int adj_stage = 0;          // adjoint convolution multiplies the staged attenuation on store and
                              // the adjoint rotation bulk-copies its (premultiplied) slices
  size_t conv_smem_adj = 0, rota_smem_stage = 0;
  int rot_nband = 0;          // bands of output rows (adj_stage 2)
  int* d_err = nullptr;       // bounded-wait give-ups
  int rotf_vpb = 1, rotf_smem_ok = 1;
  size_t rotf_smem = 0;
  int att_smem_ok = 1;
  int rota_smem_ok = 1, nsplit_adj = 1, nsplit_adj_max = 1;
  // tuned launch shapes (0 = analytic default); tuned_nv = the view count they were tuned for
  int tune_fwd_cy = 0, tune_adj_cy = 0, tune_rotf_nsplit = 0, tuned_nv = 0;
  size_t rota_smem = 0;
  // fused projector pair on z-fastest layouts (zpath.cuh): :two, attenuation
  // cache, separable PSF planes, planes that fit in shared memory
  int zpath = 0;
  ZGeom zg{};
  size_t izN = 0;              // floats of one IZ volume (L * L * nzp)
  float* d_imgIZ = nullptr;    // forward input / OS-EM iterate (IZ)
  float* d_backIZ = nullptr;   // back-projection accumulator (IZ)
  float* d_Hz = nullptr;       // [nset][ny][2 hs] pass weights
  float* d_Ez = nullptr;       // [nset][ny][2 ts] forward tails, adjoint folds
  int* d_Rz = nullptr;         // [nset][ny][8] tap-block ranges of the four passes
  double ztaps[2] = {0, 0};    // mean kept taps per plane of the fused passes (z, x)
  int zshape_fwd = -1, zshape_adj = -1;
  // large-plane kernels (zpath == 2): task width, column / row tiles, shared
  // memory and resident blocks per SM of k_zs_fz, k_zs_fx, k_zs_adj, and the
  // forward's plane-tile exchange buffer
  int zs_w = 8, zs_tx = 8, zs_tz = 4, zs_fz_nth = kZsNth / 2, zs_adj_nth = kZsNth, zs_adj_tx = 8;
  size_t zs_smem[3] = {0, 0, 0};
  int zs_occ[3] = {1, 1, 1};
  float* d_Q = nullptr;
  // split kernels with the gather rotation adjoint: the premultiplied adjoint
  // planes are transposed into d_Tz (z fastest) and gathered into d_backIZ
  int gadj = 0;
  float* d_Tz = nullptr;
  size_t zfwd_smem_b = 0, zadj_smem_b = 0;
  size_t bytes = 0;
  // stream on which the plan is built and its buffers are (de)allocated;
  // async_alloc: cudaMallocAsync/cudaFreeAsync on it (no device-wide sync)
  cudaStream_t home = 0;
  bool async_alloc = false;
  Profiler prof;
  std::mutex mu;
};

namespace {

template <class T>
int dalloc(spect_plan_s* p, T** ptr, size_t count) {
  size_t b = sizeof(T) * std::max<size_t>(count, 1);
  cudaError_t e = p->async_alloc ? cudaMallocAsync((void**)ptr, b, p->home) : cudaMalloc((void**)ptr, b);
  if (e != cudaSuccess) {
    *ptr = nullptr;
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? SPECT_ERR_OOM : SPECT_ERR_CUDA,
                std::string("cudaMalloc(") + std::to_string(b) + " bytes): " + cudaGetErrorString(e));
  }
  p->bytes += b;
  return SPECT_OK;
}

void free_plan(spect_plan_s* p) {
  void* ptrs[] = {p->d_mumap, p->d_att, p->d_err, p->d_r1view, p->d_R1, p->d_gscr_r1, p->d_H,     p->d_rot,      p->d_viewset,   p->d_tw,         p->d_all,
                  p->d_idx,   p->d_P,     p->d_part,     p->d_Vs,      p->d_imgpart,    p->d_gB,
                  p->d_gacc,  p->d_gscr_adj, p->d_views_tmp, p->d_ones, p->d_asum,       p->d_flag, p->d_sub,
                  p->d_io_img, p->d_io_views, p->d_Hsep, p->d_Tsep, p->d_imgIZ, p->d_backIZ, p->d_Hz, p->d_Ez, p->d_Tz, p->d_Rz, p->d_Q};
  for (void* q : ptrs)
    if (q) {
      if (p->async_alloc) cudaFreeAsync(q, p->home);
      else cudaFree(q);
    }
  delete p;
}

void dfree(spect_plan_s* p, void* q) {
  if (!q) return;
  if (p->async_alloc) cudaFreeAsync(q, p->home);
  else cudaFree(q);
}

// host -> device copy of a host buffer that may go away after the call
int upload(spect_plan_s* p, void* d, const void* h, size_t b) {
  cudaError_t e = cudaMemcpyAsync(d, h, b, cudaMemcpyHostToDevice, p->home);
  if (e == cudaSuccess) e = cudaStreamSynchronize(p->home);
  if (e != cudaSuccess) return fail(SPECT_ERR_CUDA, std::string("upload: ") + cudaGetErrorString(e));
  return SPECT_OK;
}

int check_launch(const char* what) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(SPECT_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return SPECT_OK;
}

// LAUNCH(plan, kind, stream, name, <kernel launch expression>)
#define LAUNCH(P, KIND, ST, NAME, ...)                   \
  do {                                                   \
    cudaEvent_t ea_ = nullptr, eb_ = nullptr;            \
    if ((P)->prof.on) {                                  \
      ea_ = (P)->prof.get();                             \
      eb_ = (P)->prof.get();                             \
      cudaEventRecord(ea_, ST);                          \
    }                                                    \
    __VA_ARGS__;                                         \
    if ((P)->prof.on) {                                  \
      cudaEventRecord(eb_, ST);                          \
      (P)->prof.pending.push_back({KIND, ea_, eb_});     \
    }                                                    \
    STATUS_TRY(check_launch(NAME));                      \
  } while (0)

// Launch configuration that depends only on the plan's sizes.
int configure(spect_plan_s* p) {
  int dev;
  CUDA_TRY(cudaGetDevice(&dev));
  p->device = dev;
  CUDA_TRY(cudaDeviceGetAttribute(&p->sm_count, cudaDevAttrMultiProcessorCount, dev));
  int optin = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  p->max_smem = (size_t)optin;
  const Geom& g = p->g;
  // ---- convolution kernels
  ConvGeom& cg = p->cg;
  cg.nx = g.nx;
  cg.ny = g.ny;
  cg.nz = g.nz;
  cg.Npx = g.Npx;
  cg.Npz = g.Npz;
  cg.logNpx = g.logNpx;
  cg.logNpz = g.logNpz;
  cg.padup = g.padup;
  cg.padleft = g.padleft;
  cg.hx = (p->px - 1) / 2;
  cg.hz = (p->pz - 1) / 2;
  cg.Q = std::max(1, g.Npz / 2);
  cg.QS = cg.Q + 1;
  cg.CX = std::min(32, g.Npx);
  cg.logCX = ilog2(cg.CX);
  cg.CZ = std::min(32, g.Npz);
  cg.logCZ = ilog2(cg.CZ);
  p->RX = g.Npx / cg.CX;
  p->RZ = g.Npz / cg.CZ;
  size_t base = (size_t)conv_tables_bytes_rt(p->RX, p->RZ);
  size_t Bb = sizeof(float2) * (size_t)g.nx * cg.QS;
  p->conv_bsmem = (base + Bb <= p->max_smem) ? 1 : 0;
  p->conv_smem = base + (p->conv_bsmem ? Bb : 0);
  int occ = 1;
  cudaError_t ce = cudaErrorInvalidValue;
  switch (p->RX) {
    case 1: ce = conv2_setup_rx1(p->RZ, p->conv_smem, &occ); break;
    case 2: ce = conv2_setup_rx2(p->RZ, p->conv_smem, &occ); break;
    case 4: ce = conv2_setup_rx4(p->RZ, p->conv_smem, &occ); break;
    case 8: ce = conv2_setup_rx8(p->RZ, p->conv_smem, &occ); break;
    case 16: ce = conv2_setup_rx16(p->RZ, p->conv_smem, &occ); break;
  }
  if (ce != cudaSuccess) return fail(SPECT_ERR_CUDA, std::string("conv kernel setup: ") + cudaGetErrorString(ce));
  p->conv_grid = p->sm_count * std::max(occ, 1);
  // plane staging of the forward kernel: B in shared memory, planes of a
  // multiple of 16 bytes, room for the staging buffers (+ attenuation)
  {
    const size_t nplane = (size_t)g.nx * g.nz;
    const size_t stage = sizeof(float) * nplane * 2 + 16;
    p->conv_stage = (p->conv_bsmem && (nplane % 4) == 0 && p->conv_smem + stage <= p->max_smem &&
                     !(std::getenv("SPECT_NO_STAGE") && std::getenv("SPECT_NO_STAGE")[0] == '1'))
                        ? 1
                        : 0;
    p->conv_smem_fwd = p->conv_smem + (p->conv_stage ? stage : 0);
  }
  if (!p->conv_bsmem) STATUS_TRY(dalloc(p, &p->d_gB, (size_t)g.nx * cg.QS * p->conv_grid));
  if (p->RX * p->RZ > 32) STATUS_TRY(dalloc(p, &p->d_gacc, (size_t)cg.Q * g.Npx * p->conv_grid));
  // ---- forward rotation
  p->rotf_vpb = std::max(1, std::min(8, 512 / g.nx));
  size_t slice = (size_t)g.nx * g.ny;
  // staged slices: image (+ mu-map when the attenuation is not cached)
  p->rotf_smem = (p->d_att ? 1 : 2) * slice * sizeof(float);
  p->rotf_smem_ok = p->rotf_smem <= p->max_smem;
  if (p->rotf_smem_ok) {
    CUDA_TRY(cudaFuncSetAttribute((const void*)k_rot_fwd<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)p->max_smem));
    CUDA_TRY(cudaFuncSetAttribute((const void*)k_rot_fwd<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)p->max_smem));
  }
  p->att_smem_ok = slice * sizeof(float) <= p->max_smem;
  if (p->att_smem_ok)
    CUDA_TRY(cudaFuncSetAttribute((const void*)k_atten_build<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->max_smem));
  // ---- adjoint rotation
  int nseg = std::max(1, kRotAdjThreads / g.nx);
  p->rota_smem = (2 * slice + (size_t)nseg * g.nx) * sizeof(float);
  p->rota_smem_ok = p->rota_smem <= p->max_smem;
  p->nsplit_adj = std::max(1, std::min(8, cdiv(2 * p->sm_count, g.nz)));
  // the autotuner may try up to 16 view splits when the split partial images stay small
  p->nsplit_adj_max = (sizeof(float) * p->N * 16 <= ((size_t)256 << 20) && p->rota_smem <= p->max_smem)
                          ? std::max(p->nsplit_adj, 16)
                          : p->nsplit_adj;
  if (p->rota_smem_ok) {
    CUDA_TRY(cudaFuncSetAttribute((const void*)k_rot_adj<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->max_smem));
    CUDA_TRY(cudaFuncSetAttribute((const void*)k_rot_adj<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->max_smem));
  } else {
    size_t per = 2 * slice + (size_t)nseg * g.nx;
    STATUS_TRY(dalloc(p, &p->d_gscr_adj, per * g.nz * p->nsplit_adj_max));
  }
  // staged adjoint (attenuation cache, :two): the adjoint convolution
  // multiplies the bulk-copied attenuation plane into its output on store, and
  // the adjoint rotation bulk-copies those premultiplied slices into two
  // shared buffers (rows of nx floats: nx a multiple of 4 for 16-byte copies)
  {
    const size_t nplane = (size_t)g.nx * g.nz;
    const size_t cadj = p->conv_smem + sizeof(float) * nplane + 16;
    const char* ns = std::getenv("SPECT_NO_STAGE");
    const bool ok = p->d_att && p->interp == SPECT_INTERP_TWO && (g.nx % 4) == 0 && cadj <= p->max_smem &&
                    !(ns && ns[0] == '1');
    // 1: whole slices (accumulator + two slices); 2: bands of output rows
    // (accumulator band + two chunks of kRotBandRows rows)
    const int as = acc_stride(g.nx);
    const size_t ptab = sizeof(float2) * (size_t)(g.nx + g.ny);  // position tables
    const size_t rsm = ((size_t)acc_floats(g.ny, as) + 2 * slice) * sizeof(float) + 16 + ptab;
    int nband = 0;
    size_t bsm = 0;
    for (int nb = 2; nb <= g.ny && ok && rsm > p->max_smem; ++nb) {
      bsm = sizeof(float) * ((size_t)acc_floats(cdiv(g.ny, nb), as) + 2 * (size_t)kRotBandRows * g.nx) + 16 + ptab;
      if (bsm <= p->max_smem) {
        nband = nb;
        break;
      }
    }
    p->adj_stage = !ok ? 0 : rsm <= p->max_smem ? 1 : nband ? 2 : 0;
    p->rot_nband = nband;
    p->conv_smem_adj = p->adj_stage ? cadj : p->conv_smem;
    p->rota_smem_stage = p->adj_stage == 1 ? rsm : bsm;
    if (p->adj_stage == 1)
      CUDA_TRY(cudaFuncSetAttribute((const void*)k_rot_adj_stream, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)p->max_smem));
    if (p->adj_stage == 2)
      CUDA_TRY(cudaFuncSetAttribute((const void*)k_rot_adj_band, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)p->max_smem));
  }
  return SPECT_OK;
}

// chunking of the depth planes for a call with nv views
// depth-chunk tile of the persistent convolution kernels: items = nv x
// ceil(ny/cy) are dealt round-robin to conv_grid CTAs, so the makespan is
// ceil(items/grid) x (cy + c0) plane costs (c0: per-item overhead, the
// chunk's inverse transforms for the forward).  The analytic choice
// minimises it; the autotuner may override it for the view count it tuned.
int best_chunk(const spect_plan_s* p, int nv, double c0) {
  double best = 1e300;
  int bc = p->ny;
  for (int cy = 1; cy <= p->ny; ++cy) {
    const int nc = cdiv(p->ny, cy);
    if (nc > p->nchunk_max) continue;
    const double waves = std::ceil((double)nv * nc / p->conv_grid);
    const double cost = waves * (cy + c0);
    if (cost < best - 1e-9) {
      best = cost;
      bc = cy;
    }
  }
  return bc;
}

void chunking(const spect_plan_s* p, int nv, bool adj, int* chunkY, int* nchunks) {
  int cy = 0;
  if (p->tuned_nv == nv) cy = adj ? p->tune_adj_cy : p->tune_fwd_cy;
  if (cy <= 0) cy = best_chunk(p, std::max(nv, 1), adj ? 0.25 : 1.0);
  *chunkY = cy;
  *nchunks = cdiv(p->ny, cy);
}

Conv2Args conv_args(const spect_plan_s* p) {
  Conv2Args a;
  std::memset(&a, 0, sizeof(a));
  a.g = p->cg;
  a.Hs = p->d_H;
  a.viewset = p->d_viewset;
  a.gB = p->d_gB;
  a.gacc = p->d_gacc;
  a.tw = p->d_tw;
  a.bsmem = p->conv_bsmem;
  // :two with the cache: the attenuation is applied inside the convolution kernels
  a.att = p->d_att;
  a.att_mul = (p->d_att && p->interp == SPECT_INTERP_TWO) ? 1 : 0;
  a.err = p->d_err;
  return a;
}

// k_sconv_fwd / k_sconv_adj instantiations, in kSepShapes order
#define SEP_SHAPES(K)                                                                                   \
  {(const void*)K<1, 512>, (const void*)K<2, 512>, (const void*)K<3, 512>, (const void*)K<4, 512>,   \
   (const void*)K<1, 640>, (const void*)K<2, 640>, (const void*)K<3, 640>, (const void*)K<1, 1024>,  \
   (const void*)K<2, 1024>}
const void* const kSconvFwd[kSepNShapes] = SEP_SHAPES(k_sconv_fwd);
const void* const kSconvAdj[kSepNShapes] = SEP_SHAPES(k_sconv_adj);
#undef SEP_SHAPES

cudaError_t sep_launch(const void* const* table, int shape, int grid, size_t smem, cudaStream_t st, SepArgs a) {
  void* args[] = {&a};
  return cudaLaunchKernel(table[shape], dim3(grid), dim3(kSepShapes[shape].nth), args, smem, st);
}

SepArgs sep_args(const spect_plan_s* p) {
  SepArgs a;
  std::memset(&a, 0, sizeof(a));
  a.nx = p->g.nx;
  a.ny = p->g.ny;
  a.nz = p->g.nz;
  a.px = p->px;
  a.pz = p->pz;
  a.att = p->d_att;
  a.att_mul = (p->d_att && p->interp == SPECT_INTERP_TWO) ? 1 : 0;
  a.H = p->d_Hsep;
  a.hs = p->sep_hs;
  a.viewset = p->d_viewset;
  a.err = p->d_err;
  return a;
}

cudaError_t conv_launch(const spect_plan_s* p, int kind, int grid, cudaStream_t st, const Conv2Args& a,
                        size_t smem = 0) {
  if (!smem) smem = p->conv_smem;
  switch (p->RX) {
    case 1: return conv2_launch_rx1(kind, p->RZ, grid, smem, st, a);
    case 2: return conv2_launch_rx2(kind, p->RZ, grid, smem, st, a);
    case 4: return conv2_launch_rx4(kind, p->RZ, grid, smem, st, a);
    case 8: return conv2_launch_rx8(kind, p->RZ, grid, smem, st, a);
    case 16: return conv2_launch_rx16(kind, p->RZ, grid, smem, st, a);
  }
  return cudaErrorInvalidValue;
}

ZArgs zargs(const spect_plan_s* p) {
  ZArgs a;
  std::memset(&a, 0, sizeof(a));
  a.g = p->zg;
  a.img = p->d_imgIZ;
  a.att = p->d_att;
  a.H = p->d_Hz;
  a.E = p->d_Ez;
  a.R = p->d_Rz;
  a.rot = p->d_rot;
  a.viewset = p->d_viewset;
  a.err = p->d_err;
  return a;
}

// zpath forward of nidx views of the IZ image: k_zfwd (rotation, attenuation,
// convolution, depth sum of chunks) then the chunk sum (+ EM ratio y/(Ax+bg))
// depth chunks of the large-plane adjoint over nv views and `tiles` column
// tiles: about four work items per SM (a short last wave), at most
// nchunk_max chunks
void zs_chunking(const spect_plan_s* p, int nv, int tiles, int* chunkY, int* nchunks) {
  int nc = std::max(1, std::min(p->ny, cdiv(4 * p->sm_count, std::max(1, nv * tiles))));
  nc = std::min(nc, (int)p->nchunk_max);
  *chunkY = cdiv(p->ny, nc);
  *nchunks = cdiv(p->ny, *chunkY);
}

int zforward(spect_plan_s* p, float* views, const float* imgIZ, const int* vidx, int nidx, cudaStream_t st,
             const float* y, const float* bg, float* partbuf, int gmax) {
  for (int g0 = 0; g0 < nidx; g0 += gmax) {
    const int nv = std::min(gmax, nidx - g0);
    const int* vi = vidx + g0;
    int cy, nc;
    ZArgs a = zargs(p);
    a.img = imgIZ;
    a.vidx = vi;
    a.nv = nv;
    a.part = partbuf;
    if (p->zpath == 2) {  // large planes: gather + z pass -> Q, x pass + depth sum -> part
      // the fused kernel's depth chunks: the same partial sums, bit for bit
      const int ntz = cdiv(p->nz, p->zs_tz);
      chunking(p, nv, false, &cy, &nc);
      a.chunkY = cy;
      a.nchunks = nc;
      a.Q = p->d_Q;
      a.tx = p->zs_tx;
      a.tz = p->zs_tz;
      const int n1 = nv * p->ny * (p->nx / p->zs_tx), n2 = nv * nc * ntz;
      LAUNCH(p, K_CONV_FWD, st, "k_zs_fz",
             zs_fz_launch(p->zs_w, p->zs_fz_nth, std::min(n1, p->sm_count * p->zs_occ[0]), p->zs_smem[0], st, a));
      LAUNCH(p, K_CONV_FWD, st, "k_zs_fx",
             zs_fx_launch(p->zs_w, std::min(n2, p->sm_count * p->zs_occ[1]), p->zs_smem[1], st, a));
    } else {
      chunking(p, nv, false, &cy, &nc);
      a.chunkY = cy;
      a.nchunks = nc;
      const int gs = std::min(p->sm_count, nv * nc);
      LAUNCH(p, K_CONV_FWD, st, "k_zfwd", zfwd_launch(p->zshape_fwd, gs, p->zfwd_smem_b, st, a));
    }
    const size_t n = (size_t)nv * p->nxz;
    const int rb = (int)std::min<size_t>((n + 255) / 256, (size_t)p->sm_count * 16);
    LAUNCH(p, K_REDUCE_VIEWS, st, "k_reduce_views",
           k_reduce_views<<<rb, 256, 0, st>>>(partbuf, nv, nc, (int)p->nxz, views + (size_t)g0 * p->nxz, y, bg, vi));
  }
  return SPECT_OK;
}

// zpath adjoint of nidx views into outIZ (IZ layout): per group k_zadj (T
// planes) then k_zrot_adj (gather over the group's views; groups after the
// first add to the accumulator).  mode 0: out = A' views; 1: zeros -> Inf;
// 2: out = x .* (A' views) ./ asum (x, asum in IZ; out may be x).
int zbackward(spect_plan_s* p, float* outIZ, const float* views, const int* vidx, int nidx, cudaStream_t st, int mode,
              const float* xIZ, const float* asumIZ) {
  if (nidx == 0) {
    CUDA_TRY(cudaMemsetAsync(outIZ, 0, sizeof(float) * p->izN, st));
    return SPECT_OK;
  }
  const int grot = std::max(1, cdiv((long long)p->nx * p->nx * 16, 256));  // 16 lanes per image column
  for (int g0 = 0; g0 < nidx; g0 += p->gmax) {
    const int nv = std::min(p->gmax, nidx - g0);
    const int* vi = vidx + g0;
    int cy, nc;
    ZArgs a = zargs(p);
    a.views = views + (size_t)g0 * p->nxz;
    a.T = p->d_P;
    a.vidx = vi;
    a.nv = nv;
    if (p->zpath == 2) {  // large planes: column tiles, x pass and z pass x attenuation -> T
      const int ntx = p->nx / p->zs_adj_tx;
      zs_chunking(p, nv, ntx, &cy, &nc);
      a.chunkY = cy;
      a.nchunks = nc;
      a.tx = p->zs_adj_tx;
      LAUNCH(p, K_CONV_ADJ, st, "k_zs_adj",
             zs_adj_launch(p->zs_w, p->zs_adj_nth, std::min(nv * ntx * nc, p->sm_count * p->zs_occ[2]),
                           p->zs_smem[2], st, a));
    } else {
      chunking(p, nv, true, &cy, &nc);
      a.chunkY = cy;
      a.nchunks = nc;
      const int gs = std::min(p->sm_count, nv * nc);
      LAUNCH(p, K_CONV_ADJ, st, "k_zadj", zadj_launch(p->zshape_adj, gs, p->zadj_smem_b, st, a));
    }
    const bool last = g0 + nv >= nidx;
    LAUNCH(p, K_ROT_ADJ, st, "k_zrot_adj",
           zrot_adj_launch(p->zg, grot, st, p->d_P, p->d_rot, vi, nv, g0 > 0 ? p->d_backIZ : nullptr,
                           last ? outIZ : p->d_backIZ, xIZ, asumIZ, last ? mode : 0));
  }
  return SPECT_OK;
}

// forward projection of nidx views (device index list vidx) into views;
// with y/bg non-null the output is the EM ratio y/(A x + bg).
int forward_scratch(spect_plan_s* p, float* views, const float* image, const int* vidx, int nidx, cudaStream_t st,
                    const float* y, const float* bg, float* Pbuf, float* partbuf, int gmax) {
  if (p->zpath) {
    LAUNCH(p, K_OTHER, st, "k_to_iz", zto_iz_launch(p->zg, st, image, p->d_imgIZ));
    return zforward(p, views, p->d_imgIZ, vidx, nidx, st, y, bg, partbuf, gmax);
  }
  const Geom& g = p->g;
  for (int g0 = 0; g0 < nidx; g0 += gmax) {
    const int nv = std::min(gmax, nidx - g0);
    const int* vi = vidx + g0;
    // rotation + attenuation -> P
    int vpb = p->rotf_vpb;
    int nsplit = std::max(1, std::min(cdiv(2 * p->sm_count, g.nz), cdiv(nv, vpb)));
    if (p->tuned_nv == nv && p->tune_rotf_nsplit > 0) nsplit = std::min(p->tune_rotf_nsplit, cdiv(nv, vpb));
    dim3 grid(g.nz, nsplit);
    const int thr = g.nx * vpb;
    const float* att = p->d_att;
    if (p->interp == SPECT_INTERP_ONE) {
      // 3-pass shear rotation of the image slices, then the attenuation
      dim3 g1(g.nz, std::min(nv, p->r1_grid_y));
      LAUNCH(p, K_ROT_FWD, st, "k_rot1_fwd",
             k_rot1_fwd<<<g1, kRot1Threads, p->r1f_smem_ok ? p->r1f_smem : 0, st>>>(
                 p->r1, image, 0, p->d_r1view, vi, nv, p->d_R1, p->r1f_smem_ok, p->d_gscr_r1));
      const size_t n = (size_t)nv * p->N;
      LAUNCH(p, K_ROT_FWD, st, "k_att_combine",
             k_att_combine<false><<<(int)std::min<size_t>((n + 255) / 256, (size_t)p->sm_count * 16), 256, 0, st>>>(
                 att, p->d_R1, vi, nv, g.nx, g.ny, g.nz, Pbuf));
    } else
    LAUNCH(p, K_ROT_FWD, st, "k_rot_fwd",
           if (p->rotf_smem_ok && att) k_rot_fwd<true, true><<<grid, thr, p->rotf_smem, st>>>(
               g, image, p->d_mumap, att, p->d_rot, vi, nv, Pbuf);
           else if (p->rotf_smem_ok) k_rot_fwd<true, false><<<grid, thr, p->rotf_smem, st>>>(
               g, image, p->d_mumap, att, p->d_rot, vi, nv, Pbuf);
           else if (att) k_rot_fwd<false, true><<<grid, thr, 0, st>>>(g, image, p->d_mumap, att, p->d_rot, vi, nv,
                                                                      Pbuf);
           else k_rot_fwd<false, false><<<grid, thr, 0, st>>>(g, image, p->d_mumap, att, p->d_rot, vi, nv,
                                                              Pbuf));
    // FFT convolution + depth sum -> part
    Conv2Args a = conv_args(p);
    int cy, nc;
    chunking(p, nv, false, &cy, &nc);
    a.P = Pbuf;
    a.vidx = vi;
    a.nv = nv;
    a.chunkY = cy;
    a.nchunks = nc;
    a.part = partbuf;
    int gridc = std::min(p->conv_grid, nv * nc);
    if (p->sep) {
      SepArgs sa = sep_args(p);
      sa.P = Pbuf;
      sa.vidx = vi;
      sa.nv = nv;
      sa.chunkY = cy;
      sa.nchunks = nc;
      sa.part = partbuf;
      const int gs = std::min(p->sm_count, nv * nc);
      const size_t sm = p->sep_fwd_smem;
      LAUNCH(p, K_CONV_FWD, st, "k_sconv_fwd", sep_launch(kSconvFwd, p->sep_shape_fwd, gs, sm, st, sa));
    } else
    LAUNCH(p, K_CONV_FWD, st, "k_conv_fwd",
           conv_launch(p, p->conv_stage ? 3 : 0, gridc, st, a, p->conv_stage ? p->conv_smem_fwd : p->conv_smem));
    // chunk sum (+ EM ratio) -> views
    size_t n = (size_t)nv * p->nxz;
    int rb = (int)std::min<size_t>((n + 255) / 256, (size_t)p->sm_count * 16);
    LAUNCH(p, K_REDUCE_VIEWS, st, "k_reduce_views",
           k_reduce_views<<<rb, 256, 0, st>>>(partbuf, nv, nc, (int)p->nxz, views + (size_t)g0 * p->nxz, y, bg,
                                              vi));
  }
  return SPECT_OK;
}

int forward(spect_plan_s* p, float* views, const float* image, const int* vidx, int nidx, cudaStream_t st,
            const float* y, const float* bg) {
  return forward_scratch(p, views, image, vidx, nidx, st, y, bg, p->d_P, p->d_part, p->gmax);
}

// back-projection of nidx views.  mode 0: image = A' views; mode 1: image =
// A' views with zeros -> Inf (EM sensitivity); mode 2: image .*= (A' views) ./ asum
int backward(spect_plan_s* p, float* image, const float* views, const int* vidx, int nidx, cudaStream_t st,
             int mode, const float* asum) {
  if (p->zpath) {
    STATUS_TRY(zbackward(p, p->d_backIZ, views, vidx, nidx, st, 0, nullptr, nullptr));
    LAUNCH(p, K_REDUCE_IMAGE, st, "k_from_iz", zfrom_iz_launch(p->zg, st, p->d_backIZ, image, asum, mode));
    return SPECT_OK;
  }
  const Geom& g = p->g;
  const int nsplit = p->nsplit_adj;
  if (nidx == 0) {
    CUDA_TRY(cudaMemsetAsync(p->d_imgpart, 0, sizeof(float) * p->N * nsplit, st));
  }
  for (int g0 = 0; g0 < nidx; g0 += p->gmax) {
    const int nv = std::min(p->gmax, nidx - g0);
    const int* vi = vidx + g0;
    Conv2Args a = conv_args(p);
    a.views = views + (size_t)g0 * p->nxz;
    a.VsOut = p->d_Vs;
    a.nv = nv;
    a.vidx = vi;
    int cy, nc;
    chunking(p, nv, true, &cy, &nc);
    if (p->sep_adj) {
      SepArgs sa = sep_args(p);
      sa.att_mul = p->adj_stage ? 1 : 0;
      sa.tails = p->d_Tsep;
      sa.ts = p->sep_ts;
      sa.views = views + (size_t)g0 * p->nxz;
      sa.T = p->d_P;
      sa.vidx = vi;
      sa.nv = nv;
      sa.chunkY = cy;
      sa.nchunks = nc;
      const int gs = std::min(p->sm_count, nv * nc);
      const size_t sm = p->sep_adj_smem;
      LAUNCH(p, K_CONV_ADJ, st, "k_sconv_adj", sep_launch(kSconvAdj, p->sep_shape_adj, gs, sm, st, sa));
    } else {
      a.vsplit = std::max(1, std::min(8, cdiv(p->conv_grid, nv)));
      LAUNCH(p, K_VSPEC, st, "k_vspec", conv_launch(p, 2, std::min(p->conv_grid, nv * a.vsplit), st, a));
      a.Vs = p->d_Vs;
      a.T = p->d_P;
      a.chunkY = cy;
      a.nchunks = nc;
      LAUNCH(p, K_CONV_ADJ, st, "k_conv_adj",
             conv_launch(p, p->adj_stage ? 4 : 1, std::min(p->conv_grid, nv * nc), st, a, p->conv_smem_adj));
    }
    dim3 grid(g.nz, nsplit);
    const size_t rsm = p->rota_smem_ok ? p->rota_smem : 0;
    if (p->gadj) {  // premultiplied planes -> z fastest -> gather into the IZ accumulator
      LAUNCH(p, K_ROT_ADJ, st, "k_t_to_z",
             zt_to_z_launch(p->zg, nv * g.ny, st, p->d_P, p->d_Tz, p->adj_stage ? nullptr : p->d_att, vi));
      const int grot = std::max(1, cdiv((long long)p->nx * p->nx * 16, 256));
      LAUNCH(p, K_ROT_ADJ, st, "k_zrot_adj",
             zrot_adj_launch(p->zg, grot, st, p->d_Tz, p->d_rot, vi, nv, g0 > 0 ? p->d_backIZ : nullptr, p->d_backIZ,
                             nullptr, nullptr, 0));
    } else if (p->interp == SPECT_INTERP_ONE) {
      const size_t n = (size_t)nv * p->N;
      LAUNCH(p, K_ROT_ADJ, st, "k_att_combine",
             k_att_combine<true><<<(int)std::min<size_t>((n + 255) / 256, (size_t)p->sm_count * 16), 256, 0, st>>>(
                 p->d_att, p->d_P, vi, nv, g.nx, g.ny, g.nz, p->d_R1));
      LAUNCH(p, K_ROT_ADJ, st, "k_rot1_adj",
             k_rot1_adj<<<grid, kRot1Threads, p->r1a_smem_ok ? p->r1a_smem : 0, st>>>(
                 p->r1, p->d_R1, p->d_r1view, vi, nv, p->d_imgpart, g0 > 0 ? 1 : 0, p->r1a_smem_ok, p->d_gscr_r1));
    } else
    LAUNCH(p, K_ROT_ADJ, st, "k_rot_adj",
           if (p->adj_stage == 2) k_rot_adj_band<<<dim3(g.nz, nsplit, p->rot_nband), kRotAdjThreads,
                                                   p->rota_smem_stage, st>>>(
               g, p->d_P, p->d_rot, vi, nv, p->d_imgpart, g0 > 0 ? 1 : 0, p->rot_nband, p->d_err);
           else if (p->adj_stage == 1) k_rot_adj_stream<<<std::min(g.nz * nsplit, p->sm_count), kRotAdjThreads,
                                                           p->rota_smem_stage, st>>>(
               g, p->d_P, p->d_rot, vi, nv, nsplit, p->d_imgpart, g0 > 0 ? 1 : 0, p->d_err);
           else if (p->d_att) k_rot_adj<true><<<grid, kRotAdjThreads, rsm, st>>>(
               g, p->d_P, p->d_mumap, p->d_att, p->d_rot, vi, nv, p->d_imgpart, g0 > 0 ? 1 : 0, p->rota_smem_ok,
               p->d_gscr_adj);
           else k_rot_adj<false><<<grid, kRotAdjThreads, rsm, st>>>(
               g, p->d_P, p->d_mumap, p->d_att, p->d_rot, vi, nv, p->d_imgpart, g0 > 0 ? 1 : 0, p->rota_smem_ok,
               p->d_gscr_adj));
  }
  if (p->gadj) {
    if (nidx == 0) CUDA_TRY(cudaMemsetAsync(p->d_backIZ, 0, sizeof(float) * p->izN, st));
    LAUNCH(p, K_REDUCE_IMAGE, st, "k_from_iz", zfrom_iz_launch(p->zg, st, p->d_backIZ, image, asum, mode));
    return SPECT_OK;
  }
  int rb = (int)std::min<size_t>((p->N + 255) / 256, (size_t)p->sm_count * 16);
  LAUNCH(p, K_REDUCE_IMAGE, st, "k_reduce_image",
         k_reduce_image<<<rb, 256, 0, st>>>(p->d_imgpart, nsplit, p->N, image, asum, mode == 2 ? 1 : 0,
                                            mode == 1 ? 1 : 0));
  return SPECT_OK;
}

int stage_index(spect_plan_s* p, const int32_t* index, int nindex, cudaStream_t st, const int** dev) {
  if (!index) {
    if (nindex != p->nview) return fail(SPECT_ERR_DIM, "DimensionMismatch: index=NULL needs nindex == nview");
    *dev = p->d_all;
    return SPECT_OK;
  }
  if (nindex < 0 || nindex > p->nview)
    return fail(SPECT_ERR_DIM, "DimensionMismatch: nindex must be in 0..nview");
  for (int i = 0; i < nindex; ++i)
    if (index[i] < 0 || index[i] >= p->nview)
      return fail(SPECT_ERR_INDEX, "BoundsError: view index " + std::to_string(index[i]) + " not in 0.." +
                                       std::to_string(p->nview - 1));
  CUDA_TRY(cudaMemcpyAsync(p->d_idx, index, sizeof(int) * nindex, cudaMemcpyHostToDevice, st));
  *dev = p->d_idx;
  return SPECT_OK;
}

int ensure_em(spect_plan_s* p, int nblocks) {
  size_t V = (size_t)p->nview * p->nxz;
  if (!p->d_views_tmp) STATUS_TRY(dalloc(p, &p->d_views_tmp, V));
  if (!p->d_ones) {
    STATUS_TRY(dalloc(p, &p->d_ones, V));
    std::vector<float> h(V, 1.0f);
    STATUS_TRY(upload(p, p->d_ones, h.data(), sizeof(float) * V));
  }
  if (!p->d_flag) STATUS_TRY(dalloc(p, &p->d_flag, 1));
  if (p->asum_blocks < nblocks) {
    const size_t unit = p->zpath ? p->izN : p->N;  // one sensitivity image
    if (p->d_asum) {
      dfree(p, p->d_asum);
      p->bytes -= sizeof(float) * unit * p->asum_blocks;
    }
    p->d_asum = nullptr;
    STATUS_TRY(dalloc(p, &p->d_asum, unit * nblocks));
    p->asum_blocks = nblocks;
  }
  return SPECT_OK;
}

__global__ void k_all_positive(const float* __restrict__ b, size_t n, int* flag) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    if (!(b[k] > 0.f)) *flag = 1;
}

int check_background(spect_plan_s* p, const float* bg, cudaStream_t st) {
  size_t V = (size_t)p->nview * p->nxz;
  CUDA_TRY(cudaMemsetAsync(p->d_flag, 0, sizeof(int), st));
  LAUNCH(p, K_OTHER, st, "k_all_positive",
         k_all_positive<<<std::max(1, std::min(cdiv(V, 256), p->sm_count * 8)), 256, 0, st>>>(bg, V, p->d_flag));
  int h = 0;
  CUDA_TRY(cudaMemcpyAsync(&h, p->d_flag, sizeof(int), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  if (h) return fail(SPECT_ERR_BACKGROUND, "need background > 0");
  return SPECT_OK;
}

// OS-EM on device buffers (mlem = one block)
// Host-side preparation of OS-EM with nblocks subsets (Ablock,
// src/ml-os-em.jl:70-84): validation, EM buffers, and the device table of
// the subsets' views (subset b = views b, b+nblocks, ... , 0-based) in
// p->d_sub.  Synchronous; nothing of it may run during a stream capture.
int prepare_osem(spect_plan_s* p, int nblocks, int niter) {
  if (nblocks < 1 || p->nview % nblocks != 0) return fail(SPECT_ERR_NBLOCKS, "nview must be divisible by nblocks!");
  if (niter < 0) return fail(SPECT_ERR_ARG, "niter must be >= 0");
  STATUS_TRY(ensure_em(p, nblocks));
  if (!p->d_sub) STATUS_TRY(dalloc(p, &p->d_sub, p->nview));
  if (p->sub_nblocks != nblocks) {
    const int nsub = p->nview / nblocks;
    std::vector<int> idx(p->nview);
    for (int b = 0; b < nblocks; ++b)
      for (int s = 0; s < nsub; ++s) idx[(size_t)b * nsub + s] = b + s * nblocks;
    STATUS_TRY(upload(p, p->d_sub, idx.data(), sizeof(int) * p->nview));
    p->sub_nblocks = nblocks;
  }
  return SPECT_OK;
}

// OS-EM enqueued on st only (no host synchronisation or host staging, so it
// can be captured into a CUDA graph); needs prepare_osem(p, nblocks) first.
int enqueue_osem(spect_plan_s* p, float* out, const float* x0, const float* y, const float* bg, int nblocks, int niter,
                 cudaStream_t st) {
  const int nsub = p->nview / nblocks;
  if (p->zpath) {  // the iterate and the sensitivities stay in the IZ layout
    LAUNCH(p, K_OTHER, st, "k_to_iz", zto_iz_launch(p->zg, st, x0, p->d_imgIZ));
    for (int b = 0; b < nblocks; ++b)
      STATUS_TRY(zbackward(p, p->d_asum + (size_t)b * p->izN, p->d_ones, p->d_sub + (size_t)b * nsub, nsub, st, 1,
                           nullptr, nullptr));
    for (int it = 0; it < niter; ++it)
      for (int b = 0; b < nblocks; ++b) {
        const int* vi = p->d_sub + (size_t)b * nsub;
        STATUS_TRY(zforward(p, p->d_views_tmp, p->d_imgIZ, vi, nsub, st, y, bg, p->d_part, p->gmax));
        STATUS_TRY(zbackward(p, p->d_imgIZ, p->d_views_tmp, vi, nsub, st, 2, p->d_imgIZ,
                             p->d_asum + (size_t)b * p->izN));
      }
    LAUNCH(p, K_REDUCE_IMAGE, st, "k_from_iz", zfrom_iz_launch(p->zg, st, p->d_imgIZ, out, nullptr, 0));
    return SPECT_OK;
  }
  for (int b = 0; b < nblocks; ++b)
    STATUS_TRY(backward(p, p->d_asum + (size_t)b * p->N, p->d_ones, p->d_sub + (size_t)b * nsub, nsub, st, 1,
                        nullptr));
  if (out != x0) CUDA_TRY(cudaMemcpyAsync(out, x0, sizeof(float) * p->N, cudaMemcpyDeviceToDevice, st));
  for (int it = 0; it < niter; ++it)
    for (int b = 0; b < nblocks; ++b) {
      const int* vi = p->d_sub + (size_t)b * nsub;
      STATUS_TRY(forward(p, p->d_views_tmp, out, vi, nsub, st, y, bg));
      STATUS_TRY(backward(p, out, p->d_views_tmp, vi, nsub, st, 2, p->d_asum + (size_t)b * p->N));
    }
  return SPECT_OK;
}

int run_osem(spect_plan_s* p, float* out, const float* x0, const float* y, const float* bg, int nblocks, int niter,
             cudaStream_t st) {
  STATUS_TRY(prepare_osem(p, nblocks, niter));
  STATUS_TRY(check_background(p, bg, st));
  return enqueue_osem(p, out, x0, y, bg, nblocks, niter, st);
}

int ensure_io(spect_plan_s* p) {
  if (!p->d_io_img) STATUS_TRY(dalloc(p, &p->d_io_img, 2 * p->N));
  if (!p->d_io_views) STATUS_TRY(dalloc(p, &p->d_io_views, 3 * (size_t)p->nview * p->nxz));
  return SPECT_OK;
}

// ------------------------------------------------------------------------
// Scratch of spect_project_static_scratch: a file-scope device array, so the
// entry point allocates nothing.  Every GPU that loads this library holds it
// until the process exits.  Host code only sees a stand-in for its name; the
// device address comes from cudaGetSymbolAddress, once per device.
constexpr size_t kStaticScratchBytes = (size_t)32 << 20;  // 32 MiB
__device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

std::mutex g_static_mu;
void* g_static_ptr[64] = {nullptr};

int static_scratch_address(void** out) {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(SPECT_ERR_UNSUPPORTED, "device index beyond 63");
  std::lock_guard<std::mutex> lk(g_static_mu);
  if (!g_static_ptr[dev]) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_scratch);
    if (e != cudaSuccess || !ptr)
      return fail(SPECT_ERR_CUDA, std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
    g_static_ptr[dev] = ptr;
  }
  *out = g_static_ptr[dev];
  return SPECT_OK;
}

// ------------------------------------------------------------------------
// Autotuner: times candidate launch shapes of the forward and adjoint
// projector for nv views on the plan's own buffers and keeps the fastest;
// results are cached per plan shape for the process.
struct TuneResult {
  int fwd_cy, adj_cy, rotf_nsplit, nsplit_adj, sep, sep_adj;
  double fwd_ms, adj_ms;
  int zshape_fwd, zshape_adj;
};
std::mutex g_tune_mu;
std::vector<std::pair<std::string, TuneResult>> g_tune_cache;

std::string tune_key(const spect_plan_s* p, int nv) {
  return std::to_string(p->nx) + "x" + std::to_string(p->nz) + "/" + std::to_string(p->px) + "x" +
         std::to_string(p->pz) + "/v" + std::to_string(p->nview) + "/n" + std::to_string(nv) + "/i" +
         std::to_string(p->interp) + "/a" + std::to_string(p->d_att ? 1 : 0) + "/d" + std::to_string(p->device) +
         "/s" + std::to_string(p->sep_fwd_ok) + std::to_string(p->sep_adj_ok) + std::to_string(p->sep_forced) +
         "/z" + std::to_string(p->zpath) + "/y" + std::to_string(p->ny);
}

bool zshape_allowed(const ZGeom& g, int i);

int time_pass(spect_plan_s* p, bool adj, int nv, int reps, double* ms) {
  cudaStream_t st = p->home;
  cudaEvent_t a, b;
  CUDA_TRY(cudaEventCreate(&a));
  CUDA_TRY(cudaEventCreate(&b));
  double best = 1e300;
  int rc = SPECT_OK;
  for (int r = 0; r <= reps && rc == SPECT_OK; ++r) {  // r = 0: warm-up
    cudaEventRecord(a, st);
    rc = adj ? backward(p, p->d_io_img, p->d_io_views, p->d_all, nv, st, 0, nullptr)
             : forward(p, p->d_io_views, p->d_io_img, p->d_all, nv, st, nullptr, nullptr);
    cudaEventRecord(b, st);
    if (cudaEventSynchronize(b) != cudaSuccess) rc = fail(SPECT_ERR_CUDA, "autotune timing");
    float t = 0;
    cudaEventElapsedTime(&t, a, b);
    if (r > 0) best = std::min(best, (double)t);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *ms = best;
  return rc;
}

int autotune(spect_plan_s* p, int nv, double* fwd_ms, double* adj_ms) {
  const std::string key = tune_key(p, nv);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (auto& kv : g_tune_cache)
      if (kv.first == key) {
        p->tuned_nv = nv;
        p->tune_fwd_cy = kv.second.fwd_cy;
        p->tune_adj_cy = kv.second.adj_cy;
        p->tune_rotf_nsplit = kv.second.rotf_nsplit;
        p->nsplit_adj = kv.second.nsplit_adj;
        p->sep = kv.second.sep && p->sep_fwd_ok;
        p->sep_adj = kv.second.sep_adj && p->sep_adj_ok;
        if (p->zpath == 1) {
          p->zshape_fwd = kv.second.zshape_fwd;
          p->zshape_adj = kv.second.zshape_adj;
        }
        *fwd_ms = kv.second.fwd_ms;
        *adj_ms = kv.second.adj_ms;
        return SPECT_OK;
      }
  }
  STATUS_TRY(ensure_io(p));
  {
    std::vector<float> h(std::max(p->N, (size_t)nv * p->nxz), 1.0f);
    STATUS_TRY(upload(p, p->d_io_img, h.data(), sizeof(float) * p->N));
    STATUS_TRY(upload(p, p->d_io_views, h.data(), sizeof(float) * (size_t)nv * p->nxz));
  }
  const bool prof = p->prof.on;
  p->prof.on = false;
  p->tuned_nv = nv;
  // candidate depth tiles: the analytic optimum for a few overhead weights
  std::vector<int> cys;
  for (double c0 : {0.0, 0.25, 0.5, 1.0, 2.0, 4.0}) {
    int c = best_chunk(p, nv, c0);
    if (std::find(cys.begin(), cys.end(), c) == cys.end()) cys.push_back(c);
  }
  if (p->zpath == 2) {
    // large-plane kernels: their tiles and chunks are fixed by the geometry;
    // the timings are recorded for the caller
    double tf = 0, ta = 0;
    int rc = time_pass(p, false, nv, 2, &tf);
    if (rc == SPECT_OK) rc = time_pass(p, true, nv, 2, &ta);
    p->prof.on = prof;
    if (rc != SPECT_OK) return rc;
    *fwd_ms = tf;
    *adj_ms = ta;
    return SPECT_OK;
  }
  if (p->zpath) {
    // fused path: depth tile and launch shape per direction
    std::vector<int> fsh, ash;
    for (int i = 0; i < kZNShapes; ++i) {
      if (!zshape_allowed(p->zg, i)) continue;
      const int cap = kZShapes[i].nt * kZShapes[i].nth, xtasks = p->nz * (p->nx / kZShapes[i].w);
      if (cap >= xtasks && cap <= 2 * xtasks && zfwd_shape_ok(i)) fsh.push_back(i);
      if (kZShapes[i].nt == 1 && kZShapes[i].nth <= 640) ash.push_back(i);
    }
    if (fsh.empty()) fsh.push_back(p->zshape_fwd);
    double bf = 1e300, ba = 1e300;
    int bcy = cys[0], bacy = cys[0], bsf = p->zshape_fwd, bsa = p->zshape_adj, rc = SPECT_OK;
    for (int sh : fsh)
      for (int cy : cys) {
        p->zshape_fwd = sh;
        p->tune_fwd_cy = cy;
        double t;
        if ((rc = time_pass(p, false, nv, 2, &t)) != SPECT_OK) break;
        if (t < bf) {
          bf = t;
          bcy = cy;
          bsf = sh;
        }
      }
    for (int sh : ash)
      for (int cy : cys) {
        if (rc != SPECT_OK) break;
        p->zshape_adj = sh;
        p->tune_adj_cy = cy;
        double t;
        if ((rc = time_pass(p, true, nv, 2, &t)) != SPECT_OK) break;
        if (t < ba) {
          ba = t;
          bacy = cy;
          bsa = sh;
        }
      }
    p->zshape_fwd = bsf;
    p->zshape_adj = bsa;
    p->tune_fwd_cy = bcy;
    p->tune_adj_cy = bacy;
    p->prof.on = prof;
    if (rc != SPECT_OK) return rc;
    *fwd_ms = bf;
    *adj_ms = ba;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache.push_back({key, TuneResult{bcy, bacy, 0, 1, p->sep, p->sep_adj, bf, ba, bsf, bsa}});
    return SPECT_OK;
  }
  // convolution kernels to try: direct (separable planes) and FFT, unless
  // SPECT_CONV fixed the choice
  std::vector<int> fconv = {p->sep}, aconv = {p->sep_adj};
  if (!p->sep_forced) {
    if (p->sep_fwd_ok) fconv = {1, 0};
    if (p->sep_adj_ok) aconv = {1, 0};
  }
  // forward: convolution kernel x depth tile x rotation split
  std::vector<int> rsplits = {0};
  for (int f : {1, 2, 4, 8})
    if (f * p->g.nz <= 8 * p->sm_count) rsplits.push_back(f);
  double bf = 1e300;
  int bcy = cys[0], brs = 0, bsep = p->sep, rc = SPECT_OK;
  for (int sp : fconv)
    for (int cy : cys)
      for (int rs : rsplits) {
        if (rc != SPECT_OK) break;
        p->sep = sp;
        p->tune_fwd_cy = cy;
        p->tune_rotf_nsplit = rs;
        double t;
        if ((rc = time_pass(p, false, nv, 2, &t)) != SPECT_OK) break;
        if (t < bf) {
          bf = t;
          bcy = cy;
          brs = rs;
          bsep = sp;
        }
      }
  p->sep = bsep;
  p->tune_fwd_cy = bcy;
  p->tune_rotf_nsplit = brs;
  // adjoint: convolution kernel x depth tile x view split of the rotation adjoint
  double ba = 1e300;
  int bacy = cys[0], bns = p->nsplit_adj, basep = p->sep_adj;
  for (int sp : aconv)
    for (int cy : cys)
      for (int ns : {1, 2, 4, 8, 16}) {
        if (rc != SPECT_OK || ns > p->nsplit_adj_max) break;
        p->sep_adj = sp;
        p->tune_adj_cy = cy;
        p->nsplit_adj = ns;
        double t;
        if ((rc = time_pass(p, true, nv, 2, &t)) != SPECT_OK) break;
        if (t < ba) {
          ba = t;
          bacy = cy;
          bns = ns;
          basep = sp;
        }
      }
  p->sep_adj = basep;
  p->tune_adj_cy = bacy;
  p->nsplit_adj = bns;
  p->prof.on = prof;
  if (rc != SPECT_OK) return rc;
  *fwd_ms = bf;
  *adj_ms = ba;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_cache.push_back({key, TuneResult{bcy, bacy, brs, bns, bsep, basep, bf, ba, -1, -1}});
  return SPECT_OK;
}

}  // namespace

// ------------------------------------------------------------------------
// Batched OS-EM: many reconstructions (one plan each, uneven sizes) enqueued
// on one non-blocking stream per job and captured into a single CUDA graph;
// spect_batch_run launches that graph once.
struct spect_batch_s {
  std::vector<spect_plan_s*> plans;
  std::vector<int> nblocks, niter;
  std::vector<float*> out;
  std::vector<const float*> x0, y, bg;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> done;
  cudaStream_t root = nullptr;
  cudaEvent_t fork = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  unsigned long long nkernels = 0;  // kernels in the graph
  bool dirty = true;
  std::mutex mu;
};

namespace {
void batch_release_graph(spect_batch_s* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

int batch_capture(spect_batch_s* b) {
  batch_release_graph(b);
  const int nj = (int)b->plans.size();
  for (int j = 0; j < nj; ++j)
    if (!b->out[j] || !b->x0[j] || !b->y[j] || !b->bg[j])
      return fail(SPECT_ERR_ARG, "spect_batch_run: job " + std::to_string(j) + " has no data");
  std::vector<char> prof(nj);
  for (int j = 0; j < nj; ++j) {
    prof[j] = b->plans[j]->prof.on;
    b->plans[j]->prof.on = false;  // no event bracketing inside the graph
  }
  CUDA_TRY(cudaStreamBeginCapture(b->root, cudaStreamCaptureModeThreadLocal));
  const unsigned long long l0 = g_launches.load();
  int rc = SPECT_OK;
  cudaError_t e = cudaEventRecord(b->fork, b->root);
  for (int j = 0; j < nj && rc == SPECT_OK && e == cudaSuccess; ++j) {
    e = cudaStreamWaitEvent(b->streams[j], b->fork, 0);
    if (e != cudaSuccess) break;
    rc = enqueue_osem(b->plans[j], b->out[j], b->x0[j], b->y[j], b->bg[j], b->nblocks[j], b->niter[j],
                      b->streams[j]);
    if (rc == SPECT_OK) e = cudaEventRecord(b->done[j], b->streams[j]);
    if (rc == SPECT_OK && e == cudaSuccess) e = cudaStreamWaitEvent(b->root, b->done[j], 0);
  }
  cudaGraph_t g = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(b->root, &g);
  // captured kernels are counted when the graph runs, not here
  b->nkernels = g_launches.load() - l0;
  g_launches.fetch_sub(b->nkernels);
  for (int j = 0; j < nj; ++j) b->plans[j]->prof.on = prof[j];
  if (rc != SPECT_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return fail(SPECT_ERR_CUDA, std::string("batch capture: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
  }
  b->graph = g;
  CUDA_TRY(cudaGraphInstantiate(&b->exec, g, 0));
  b->dirty = false;
  return SPECT_OK;
}
}  // namespace

// ====================================================================== ABI
extern "C" {

const char* spect_last_error(void) { return g_err.c_str(); }

int spect_device_info(int* sm_count, size_t* total_mem) {
  int dev;
  CUDA_TRY(cudaGetDevice(&dev));
  if (sm_count) CUDA_TRY(cudaDeviceGetAttribute(sm_count, cudaDevAttrMultiProcessorCount, dev));
  if (total_mem) {
    size_t f, t;
    CUDA_TRY(cudaMemGetInfo(&f, &t));
    *total_mem = t;
  }
  return SPECT_OK;
}

}  // extern "C"

namespace {
struct PlanOpts {
  cudaStream_t home = 0;
  bool async_alloc = false;
  int gmax_cap = 0;     // > 0: at most this many views per group (scratch bound)
  int atten_cache = -1; // -1 auto, 0 off (:two only), 1 on
  // compact PSFs: psfs holds nset distinct [ny][pz][px] stacks and
  // view_set[v] names the stack of view v (already checked for symmetry)
  const int* view_set = nullptr;
  int nset = 0;
  // Gaussian PSFs generated on the device (psfs unused): FWHM ranges along y
  bool gauss = false;
  double gx0 = 0, gx1 = 0, gz0 = 0, gz1 = 0;
};

// distinct PSF stacks of nview views (stack = ny*pp floats each): view_set[v]
// is the index into uniq (the first view of each distinct stack)
void psf_sets(const float* psfs, int nview, size_t stack, std::vector<int>& view_set, std::vector<int>& uniq) {
  view_set.assign(nview, 0);
  uniq.clear();
  for (int v = 0; v < nview; ++v) {
    int found = -1;
    for (size_t u = 0; u < uniq.size(); ++u)
      if (std::memcmp(psfs + (size_t)uniq[u] * stack, psfs + (size_t)v * stack, sizeof(float) * stack) == 0) {
        found = (int)u;
        break;
      }
    if (found < 0) {
      found = (int)uniq.size();
      uniq.push_back(v);
    }
    view_set[v] = found;
  }
}

// every px x pz plane of the given stacks point-symmetric (src/spectplan.jl:84-88)
bool psf_symmetric(const float* psfs, const std::vector<int>& stacks, size_t ny, size_t pp) {
  for (int u : stacks)
    for (size_t y = 0; y < ny; ++y) {
      const float* k = psfs + ((size_t)u * ny + y) * pp;
      for (size_t i = 0; i < pp / 2; ++i)
        if (!(k[i] == k[pp - 1 - i])) return false;
      if (!(k[pp / 2] == k[pp / 2])) return false;  // a NaN centre is not symmetric
    }
  return true;
}

// Factor every plane of the distinct PSF stacks as h[i, j] = a[i] b[j]
// (rank 1 within 1e-6 of max|h|: true for psf_gauss planes), into fa
// [set][y][px] and fb [set][y][pz] (double); Gaussian plans take the exact
// 1-D factors.  False when some plane is not separable.
bool factor_planes(const float* psfs, const std::vector<int>& uniq, int ny, int px, int pz, const PlanOpts& opts,
                   std::vector<double>& fa, std::vector<double>& fb) {
  const size_t pp = (size_t)px * pz;
  fa.assign(uniq.size() * ny * px, 0.0);
  fb.assign(uniq.size() * ny * pz, 0.0);
  auto gauss_taps = [](int n, double fwhm, double* w) {
    const int h = (n - 1) / 2;
    if (fwhm == 0) {
      for (int i = 0; i < n; ++i) w[i] = (i == h) ? 1.0 : 0.0;
      return;
    }
    const double sigma = fwhm / std::sqrt(std::log(256.0));
    double s = 0;
    for (int i = 0; i < n; ++i) {
      const double q = (double)(i - h) / sigma;
      w[i] = std::exp(-0.5 * q * q);
      s += w[i];
    }
    for (int i = 0; i < n; ++i) w[i] /= s;
  };
  for (size_t u = 0; u < uniq.size(); ++u)
    for (int y = 0; y < ny; ++y) {
      double* a = fa.data() + (u * ny + y) * px;
      double* b = fb.data() + (u * ny + y) * pz;
      if (opts.gauss) {
        auto fw = [&](double f0, double f1) { return ny <= 1 ? f0 : (y == ny - 1 ? f1 : f0 + y * ((f1 - f0) / (ny - 1))); };
        gauss_taps(px, fw(opts.gx0, opts.gx1), a);
        gauss_taps(pz, fw(opts.gz0, opts.gz1), b);
        continue;
      }
      const float* k = psfs + ((size_t)uniq[u] * ny + y) * pp;  // k[i + px j]
      const int i0 = (px - 1) / 2, j0 = (pz - 1) / 2;
      const double c = k[i0 + (size_t)px * j0];
      double mx = 0;
      for (size_t e = 0; e < pp; ++e) mx = std::max(mx, (double)std::fabs(k[e]));
      if (!(c != 0.0) || !(mx > 0.0)) return false;
      for (int i = 0; i < px; ++i) a[i] = k[i + (size_t)px * j0];
      for (int j = 0; j < pz; ++j) b[j] = k[i0 + (size_t)px * j] / c;
      double res = 0;
      for (int j = 0; j < pz; ++j)
        for (int i = 0; i < px; ++i) res = std::max(res, std::fabs(k[i + (size_t)px * j] - a[i] * b[j]));
      if (res > 1e-6 * mx) return false;
    }
  return true;
}

// adjoint folds of a centred factor w (2h + 1 taps): cL_k = sum_{d>k} w(d),
// cR_k = sum_{d<-k} w(d), k < h
void fold_tails(const double* w, int h, float* L, float* R) {
  for (int k = 0; k < h; ++k) {
    double l = 0, r = 0;
    for (int i = h + k + 1; i <= 2 * h; ++i) l += w[i];
    for (int i = 0; i < h - k; ++i) r += w[i];
    L[k] = (float)l;
    R[k] = (float)r;
  }
}

// forward clamp tails of the reversed factor wr[m] = w[p - 1 - m]:
// EL[i] = sum_{m < h - i} wr[m] (i < h), ER[k] = sum_{m > h + k} wr[m] (k < h)
void clamp_tails(const double* w, int p, float* EL, float* ER) {
  const int h = (p - 1) / 2;
  for (int i = 0; i < h; ++i) {
    double l = 0, r = 0;
    for (int m = 0; m < h - i; ++m) l += w[p - 1 - m];
    for (int m = h + 1 + i; m < p; ++m) r += w[p - 1 - m];
    EL[i] = (float)l;
    ER[i] = (float)r;
  }
}

// Zero the outer taps of a factor while their summed magnitude, per side,
// stays within 2^-27 of the factor's: below Float32 resolution of every
// output (the two sides and two factors of a plane leave out at most 2^-25 of
// its mass, against the 2^-24 rounding of one Float32 operation).
// SPECT_ZTRIM=0 keeps every tap.
void trim_taps(double* w, int n) {
  double s = 0;
  for (int i = 0; i < n; ++i) s += std::fabs(w[i]);
  const double lim = std::ldexp(s, -27);
  double acc = 0;
  for (int i = 0; i < n; ++i) {
    acc += std::fabs(w[i]);
    if (acc > lim) break;
    w[i] = 0;
  }
  acc = 0;
  for (int i = n - 1; i >= 0; --i) {
    acc += std::fabs(w[i]);
    if (acc > lim) break;
    w[i] = 0;
  }
}

// taps of a pass row w[0, len) (len a multiple of 8) that a window pass runs:
// 8-tap blocks from a 4-tap boundary, (first 4-tap block b4, block count n8)
// covering every nonzero tap, 4 b4 + 8 n8 <= len
void tap_range(const float* w, int len, int* b4, int* n8) {
  int lo = 0, hi = len - 1;
  while (lo < len && w[lo] == 0.f) ++lo;
  while (hi > lo && w[hi] == 0.f) --hi;
  if (lo >= len) {  // no tap (cannot happen for a plane factor)
    *b4 = 0;
    *n8 = 0;
    return;
  }
  int b = lo / 4, n = (hi + 1 - 4 * b + 7) / 8;
  if (4 * b + 8 * n > len) --b;  // 4 past the end: start 4 taps earlier (zeros)
  *b4 = b;
  *n8 = n;
}

// zpath launch shapes (no 1024-thread shape: it leaves too few registers):
// forward -- the fewest thread slots holding every x task of a plane (ties:
// more threads); adjoint -- the least padded x and z passes, one task per
// thread and pass
// tiles of the large-plane kernels: task width w (16 where it divides nx,
// SPECT_ZW=8 forces 8), column tile tx (32, 16 or 8 dividing nx), row tile
// tz (a multiple of 4: one x task of w outputs per thread of k_zs_fx,
// tz * nx / w <= kZsNthX); false when a kernel's shared memory does not fit
bool zs_tiles(const ZGeom& g, size_t optin, ZsTiles* t) {
  const char* e = std::getenv("SPECT_ZW");
  t->w = (g.nx % 16 == 0 && !(e && std::atoi(e) == 8)) ? 16 : 8;
  t->tx = g.nx % 32 == 0 ? 32 : (g.nx % 16 == 0 ? 16 : 8);
  t->tz = std::min(kZsNthX * t->w / g.nx / 4 * 4, zround(g.nz, 4));
  if (t->tz < 4) return false;
  return zs_fz_smem(g, t->tx) <= optin && zs_fx_smem(g, t->tz) <= optin && zs_adj_smem(g, t->tx) <= optin;
}

// shapes allowed by the geometry and by SPECT_ZW=8|16 (fixes the task width)
bool zshape_allowed(const ZGeom& g, int i) {
  const char* e = std::getenv("SPECT_ZW");
  const int force = e ? std::atoi(e) : 0;
  return zshape_fits(g, i) && (force == 0 || kZShapes[i].w == force);
}
// forward: the widest tasks, then the least thread capacity holding all x
// tasks (their outputs stay in registers), then more threads
int zpick_fwd(const ZGeom& g) {
  int best = -1;
  for (int i = 0; i < kZNShapes; ++i) {
    if (!zfwd_shape_ok(i) || !zshape_allowed(g, i)) continue;
    const ZShape& s = kZShapes[i];
    const int cap = s.nt * s.nth;
    if (cap < g.nz * (g.nx / s.w)) continue;
    if (best < 0) {
      best = i;
      continue;
    }
    const ZShape& b = kZShapes[best];
    if (s.w > b.w || (s.w == b.w && (cap < b.nt * b.nth || (cap == b.nt * b.nth && s.nth > b.nth)))) best = i;
  }
  return best;
}
// adjoint: one task per thread per pass round; the least padded work in
// 8-output units (x and z tasks, rounded up to whole rounds), wider tasks on
// ties
int zpick_adj(const ZGeom& g) {
  int best = -1;
  long long bc = 0;
  for (int i = 0; i < kZNShapes; ++i) {
    const ZShape& s = kZShapes[i];
    if (s.nt != 1 || s.nth > 640 || !zshape_allowed(g, i)) continue;
    const long long xt = (long long)g.nz * (g.nx / s.w), zt = (long long)g.nx * ((g.nz + s.w - 1) / s.w);
    const long long c = s.nth * ((xt + s.nth - 1) / s.nth + (zt + s.nth - 1) / s.nth) * (s.w / 8);
    if (best < 0 || c < bc || (c == bc && s.w > kZShapes[best].w)) {
      best = i;
      bc = c;
    }
  }
  return best;
}

int plan_create_impl(spect_plan_t* out, int nx, int ny, int nz, int px, int pz, int nview, const float* mumap,
                     const float* psfs, float dy, const float* viewangle, int interpmeth, int mode, int nthread,
                     int nthreads, const PlanOpts& opts) {
  if (!out || !mumap || (!psfs && !opts.gauss)) return fail(SPECT_ERR_ARG, "null pointer argument");
  *out = nullptr;
  if (nx <= 0 || ny <= 0 || nz <= 0 || px <= 0 || pz <= 0 || nview <= 0)
    return fail(SPECT_ERR_ARG, "sizes must be positive");
  // validation in the reference's order (src/spectplan.jl:76-93)
  if (nx != ny) return fail(SPECT_ERR_NX_NE_NY, "nx != ny");
  if ((nx % 2) || (ny % 2)) return fail(SPECT_ERR_NX_ODD, "nx odd");
  if (!(px % 2) || !(pz % 2)) return fail(SPECT_ERR_PSF_NOT_ODD, "non-odd size psfs");
  const size_t pp = (size_t)px * pz;
  // distinct PSF stacks first: identical stacks are symmetric together
  const size_t stack = (size_t)ny * pp;
  std::vector<int> view_set, uniq;
  if (opts.gauss) {  // one generated stack for every view (symmetric by construction)
    view_set.assign(nview, 0);
    uniq.push_back(0);
  } else if (opts.view_set) {
    view_set.assign(opts.view_set, opts.view_set + nview);
    for (int u = 0; u < opts.nset; ++u) uniq.push_back(u);  // stack u of the compact array
  } else {
    psf_sets(psfs, nview, stack, view_set, uniq);
    if (!psf_symmetric(psfs, uniq, ny, pp)) return fail(SPECT_ERR_PSF_ASYM, "asym. psf");
  }
  if (interpmeth != SPECT_INTERP_ONE && interpmeth != SPECT_INTERP_TWO)
    return fail(SPECT_ERR_INTERP, "bad interpmeth");
  if (nthread != nthreads) return fail(SPECT_ERR_NTHREAD, "bad nthread");
  if (mode != SPECT_MODE_FAST && mode != SPECT_MODE_MEM) return fail(SPECT_ERR_MODE, "bad mode");
  const int Npx = power2(nx + px - 1), Npz = power2(nz + pz - 1);
  if (Npx > SPECT_TW_N || Npz > SPECT_TW_N || nx > 512)
    return fail(SPECT_ERR_UNSUPPORTED, "padded plane " + std::to_string(Npx) + "x" + std::to_string(Npz) +
                                           " exceeds this build's FFT limit of " + std::to_string(SPECT_TW_N));

  spect_plan_s* p = new spect_plan_s;
  p->home = opts.home;
  p->async_alloc = opts.async_alloc;
  p->nx = nx;
  p->ny = ny;
  p->nz = nz;
  p->px = px;
  p->pz = pz;
  p->nview = nview;
  p->interp = interpmeth;
  p->mode = mode;
  p->nthread = nthread;
  p->dy = dy;
  p->N = (size_t)nx * ny * nz;
  p->nxz = (size_t)nx * nz;
  Geom& g = p->g;
  g.nx = nx;
  g.ny = ny;
  g.nz = nz;
  g.Npx = Npx;
  g.Npz = Npz;
  g.logNpx = ilog2(Npx);
  g.logNpz = ilog2(Npz);
  g.Hz = Npz / 2 + 1;
  g.padup = (Npx - nx + 1) / 2;
  g.padleft = (Npz - nz + 1) / 2;
  g.dy = dy;
  g.c0 = (float)((nx - 1) * 0.5);
  auto bail = [&](int st) {
    free_plan(p);
    return st;
  };
  // separable PSF planes (host factorisation) and the fused-path decision:
  // :two, separable planes, attenuation cache, planes that fit in shared memory
  std::vector<double> fa, fb;
  const bool sep_host = factor_planes(psfs, uniq, ny, px, pz, opts, fa, fb);
  const char* conv_env = std::getenv("SPECT_CONV");
  const bool only_fft = conv_env && std::strcmp(conv_env, "fft") == 0;
  const int pad_rot = (int)std::ceil(1.0 + nx * std::sqrt(2.0) / 2.0 - nx / 2.0);
  const ZGeom zg = zgeom_make(nx, ny, nz, px, pz, pad_rot);
  // zkind 1: the fused pair; 2: the large-plane kernels on the same layouts
  // (planes too large for the fused kernels' shared memory; SPECT_ZSTRIP=1
  // prefers them, =0 never takes them); 0: the split kernels
  int zkind = 0;
  ZsTiles zt{};
  {
    int dev = 0, optin = 0;
    const char* zenv = std::getenv("SPECT_ZPATH");
    const char* senv = std::getenv("SPECT_ZSTRIP");
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess &&
        interpmeth == SPECT_INTERP_TWO && sep_host && !only_fft && !(zenv && zenv[0] == '0') && nx % 8 == 0 &&
        zg.zpw <= 72 && zg.xpw <= 72 &&  // pass rows of at most 9 blocks of 8 taps
        zg.nzp <= 256 && opts.atten_cache != 0) {
      const bool fused = zpick_fwd(zg) >= 0 && zpick_adj(zg) >= 0 && zfwd_smem(zg, 1) <= (size_t)optin &&
                         zadj_smem(zg, 1) <= (size_t)optin;
      const bool strip = zs_tiles(zg, (size_t)optin, &zt);
      if (fused && !(senv && senv[0] == '1')) zkind = 1;
      else if (strip && !(senv && senv[0] == '0')) zkind = 2;
      else if (fused) zkind = 1;
    }
    cudaGetLastError();
  }
  const bool zcand = zkind != 0;
  // attenuation cache: on when it fits a quarter of the free device memory
  // (and 32 GiB); SPECT_ATTEN_CACHE=0 turns it off (and with it the fused
  // path).  The fused path keeps it z-fastest ([view][y][x][nzp]), the
  // other kernels as [view][y][z][x].
  {
    const char* env = std::getenv("SPECT_ATTEN_CACHE");
    const size_t cnt = zcand ? (size_t)nview * ny * nx * zg.nzp : p->N * (size_t)nview;
    size_t need = sizeof(float) * cnt, fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      cudaGetLastError();
      fr = 0;
    }
    bool want = !(env && env[0] == '0') && need <= std::min(fr / 4, (size_t)32 << 30);
    if (opts.atten_cache >= 0) want = opts.atten_cache == 1;
    if (interpmeth == SPECT_INTERP_ONE) {
      // the :one path reads its attenuation from the cache
      int st1 = dalloc(p, &p->d_att, p->N * (size_t)nview);
      if (st1 != SPECT_OK) return bail(st1);
    } else if (want && dalloc(p, &p->d_att, cnt) != SPECT_OK) {
      p->d_att = nullptr;
      g_err.clear();
    }
    p->zpath = (zcand && p->d_att) ? zkind : 0;
  }
  int st = configure(p);
  if (st != SPECT_OK) return bail(st);
  if (p->zpath == 2) {
    p->zg = zg;
    p->izN = (size_t)zg.L * zg.L * zg.nzp;
    p->zs_w = zt.w;
    p->zs_tx = zt.tx;
    p->zs_tz = zt.tz;
    p->zs_smem[0] = zs_fz_smem(zg, zt.tx);
    p->zs_smem[1] = zs_fx_smem(zg, zt.tz);
    // k_zs_fz: 256 threads, two blocks per SM (SPECT_ZS_FZ_THREADS=512: one of 512)
    const char* fz_env = std::getenv("SPECT_ZS_FZ_THREADS");
    p->zs_fz_nth = (fz_env && std::atoi(fz_env) == kZsNth) ? kZsNth : kZsNth / 2;
    // k_zs_adj: 512 threads on tiles of tx columns (SPECT_ZS_ADJ_THREADS=256:
    // 256 threads on tiles of half the width, two blocks per SM where they fit)
    const char* adj_env = std::getenv("SPECT_ZS_ADJ_THREADS");
    p->zs_adj_nth = kZsNth;
    p->zs_adj_tx = zt.tx;
    if (adj_env && std::atoi(adj_env) == kZsNth / 2 && zt.tx / 2 >= zt.w && zt.tx % 2 == 0 && (zt.tx / 2) % 4 == 0) {
      p->zs_adj_nth = kZsNth / 2;
      p->zs_adj_tx = zt.tx / 2;
    }
    p->zs_smem[2] = zs_adj_smem(zg, p->zs_adj_tx);
    cudaError_t ze = zstrip_setup((int)p->max_smem);
    if (ze == cudaSuccess) ze = zstrip_occupancy(zt.w, p->zs_fz_nth, p->zs_adj_nth, p->zs_smem, p->zs_occ);
    if (ze != cudaSuccess) return bail(fail(SPECT_ERR_CUDA, std::string("large-plane kernel setup: ") + cudaGetErrorString(ze)));
  }
  if (p->zpath == 1) {
    p->zg = zg;
    p->izN = (size_t)zg.L * zg.L * zg.nzp;
    p->zshape_fwd = zpick_fwd(zg);
    p->zshape_adj = zpick_adj(zg);
    // double-buffered adjoint x pass where it fits (SPECT_ZADJ_BUFFERS=1: one buffer)
    const char* nwa_env = std::getenv("SPECT_ZADJ_BUFFERS");
    p->zg.nwa = (zadj_smem(zg, 2) <= p->max_smem && !(nwa_env && nwa_env[0] == '1')) ? 2 : 1;
    // one forward staging buffer (SPECT_ZFWD_STAGES=2: two where they fit;
    // measured slower at 128x128x80: the shared-memory carve-out takes L1
    // from the gather's image reads)
    const char* nsf_env = std::getenv("SPECT_ZFWD_STAGES");
    p->zg.nsf = (zfwd_smem(zg, 2) <= p->max_smem && nsf_env && nsf_env[0] == '2') ? 2 : 1;
    p->zfwd_smem_b = zfwd_smem(p->zg, p->zg.nsf);
    p->zadj_smem_b = zadj_smem(p->zg, p->zg.nwa);
    const cudaError_t ze = zpath_setup((int)p->max_smem);
    if (ze != cudaSuccess) return bail(fail(SPECT_ERR_CUDA, std::string("fused kernel setup: ") + cudaGetErrorString(ze)));
  }

  // angles: default (0:nview-1)/nview * Float32(2pi), element rounded to Float32
  p->angles.resize(nview);
  const double t2pi = (double)(float)kTwoPi;
  for (int v = 0; v < nview; ++v) p->angles[v] = viewangle ? viewangle[v] : (float)((double)v / nview * t2pi);
  std::vector<float4> rot(nview);
  for (int v = 0; v < nview; ++v) {
    double phi = kTwoPi - (double)p->angles[v];
    bool ident = std::fmod((double)p->angles[v], kTwoPi) == 0.0;
    rot[v] = make_float4((float)std::cos(phi), (float)std::sin(phi), ident ? 1.f : 0.f, p->angles[v]);
  }
  p->view_set = view_set;
  p->nset = (int)uniq.size();

  // group size: rotated-plane scratch bounded by ~1 GiB
  // (the fused path's adjoint planes T hold nzp >= nz values per column)
  const size_t budget = (size_t)1 << 30;
  const size_t slot = p->zpath ? (size_t)ny * nx * zg.nzp : p->N;
  if (p->zpath) p->nsplit_adj = p->nsplit_adj_max = 1;  // no split partial images
  p->gmax = (int)std::max<size_t>(1, std::min<size_t>((size_t)nview, budget / (sizeof(float) * slot)));
  if (opts.gmax_cap > 0) p->gmax = std::min(p->gmax, opts.gmax_cap);

  if ((st = dalloc(p, &p->d_mumap, p->N)) || (st = dalloc(p, &p->d_rot, nview)) ||
      (st = dalloc(p, &p->d_viewset, nview)) || (st = dalloc(p, &p->d_tw, SPECT_TW_N)) ||
      (st = dalloc(p, &p->d_all, nview)) || (st = dalloc(p, &p->d_idx, nview)) || (st = dalloc(p, &p->d_err, 1)) ||
      (st = (cudaMemsetAsync(p->d_err, 0, sizeof(int), p->home) == cudaSuccess) ? SPECT_OK
                                                                                 : fail(SPECT_ERR_CUDA, "memset")) ||
      (st = dalloc(p, &p->d_H, (size_t)p->nset * ny * (p->cg.Q + 1) * Npx)) ||
      (st = dalloc(p, &p->d_P, (size_t)p->gmax * slot)) ||
      (st = ((p->nchunk_max = ((size_t)p->gmax * 32 * p->nxz * 4 <= ((size_t)256 << 20)) ? 32 : 16),
             dalloc(p, &p->d_part, (size_t)p->gmax * p->nchunk_max * p->nxz))) ||
      (st = dalloc(p, &p->d_Vs, (size_t)p->gmax * p->cg.Q * Npx)) ||
      (st = dalloc(p, &p->d_imgpart, (size_t)p->nsplit_adj_max * p->N)))
    return bail(st);
  {  // split kernels with the attenuation cache (:two): rotation adjoint by the
     // gather kernel, the attenuation applied by the convolution's store or by
     // the transpose (SPECT_GADJ=0 keeps the scatter kernels)
    const char* genv = std::getenv("SPECT_GADJ");
    if (!p->zpath && p->d_att && interpmeth == SPECT_INTERP_TWO && zg.nzp <= 256 && !(genv && genv[0] == '0')) {
      p->gadj = 1;
      p->zg = zg;
      p->izN = (size_t)zg.L * zg.L * zg.nzp;
      if ((st = dalloc(p, &p->d_backIZ, p->izN)) ||
          (st = dalloc(p, &p->d_Tz, (size_t)p->gmax * ny * nx * zg.nzp)))
        return bail(st);
      if (cudaMemsetAsync(p->d_backIZ, 0, sizeof(float) * p->izN, p->home) != cudaSuccess)
        return bail(fail(SPECT_ERR_CUDA, "memset"));
    }
  }
  if (p->zpath) {  // IZ volumes (zero ring and z padding) and zeroed adjoint planes
    if ((st = dalloc(p, &p->d_imgIZ, p->izN)) || (st = dalloc(p, &p->d_backIZ, p->izN)))
      return bail(st);
    if (p->zpath == 2 && (st = dalloc(p, &p->d_Q, (size_t)p->gmax * slot)))  // plane tiles of the large-plane kernels
      return bail(st);
    cudaError_t e = cudaMemsetAsync(p->d_imgIZ, 0, sizeof(float) * p->izN, p->home);
    if (e == cudaSuccess) e = cudaMemsetAsync(p->d_backIZ, 0, sizeof(float) * p->izN, p->home);
    if (e == cudaSuccess) e = cudaMemsetAsync(p->d_P, 0, sizeof(float) * (size_t)p->gmax * slot, p->home);
    if (e != cudaSuccess) return bail(fail(SPECT_ERR_CUDA, std::string("memset: ") + cudaGetErrorString(e)));
  }

  std::vector<float2> tw(SPECT_TW_N);
  for (int m = 0; m < SPECT_TW_N; ++m) {
    double a = -kTwoPi * m / SPECT_TW_N;
    tw[m] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  std::vector<int> all(nview);
  for (int v = 0; v < nview; ++v) all[v] = v;
  auto up = [&](void* d, const void* h, size_t b) -> int { return upload(p, d, h, b); };
  const cudaStream_t hs = p->home;
  if ((st = up(p->d_mumap, mumap, sizeof(float) * p->N)) || (st = up(p->d_rot, rot.data(), sizeof(float4) * nview)) ||
      (st = up(p->d_viewset, p->view_set.data(), sizeof(int) * nview)) ||
      (st = up(p->d_tw, tw.data(), sizeof(float2) * SPECT_TW_N)) ||
      (st = up(p->d_all, all.data(), sizeof(int) * nview)))
    return bail(st);

  if (interpmeth == SPECT_INTERP_ONE) {
    // Rot1 geometry and per-view shear parameters (src/rotatez.jl:249-272)
    const int pad1 = (int)std::ceil(1.0 + nx * std::sqrt(2.0) / 2.0 - nx / 2.0);
    p->r1 = Rot1Geom{nx, ny, nz, nx + 2 * pad1, pad1, nx + 2 * pad1 + 1};
    const int L = p->r1.L;
    p->r1f_smem = sizeof(float) * ((size_t)p->r1.LS * L + (size_t)kRot1Warps * L);
    p->r1a_smem = p->r1f_smem + sizeof(float) * (size_t)nx * nx;
    p->r1f_smem_ok = p->r1f_smem <= p->max_smem;
    p->r1a_smem_ok = p->r1a_smem <= p->max_smem;
    if (p->r1f_smem_ok &&
        cudaFuncSetAttribute((const void*)k_rot1_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->max_smem) != cudaSuccess)
      return bail(fail(SPECT_ERR_CUDA, "k_rot1_fwd shared memory"));
    if (p->r1a_smem_ok &&
        cudaFuncSetAttribute((const void*)k_rot1_adj, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p->max_smem) != cudaSuccess)
      return bail(fail(SPECT_ERR_CUDA, "k_rot1_adj shared memory"));
    p->r1_grid_y = std::max(1, cdiv(4 * p->sm_count, nz));
    size_t gs = 0;
    if (!p->r1f_smem_ok) gs = std::max(gs, (size_t)nz * p->r1_grid_y * (p->r1f_smem / sizeof(float)));
    if (!p->r1a_smem_ok) gs = std::max(gs, (size_t)nz * p->nsplit_adj_max * (p->r1a_smem / sizeof(float)));
    if (gs && (st = dalloc(p, &p->d_gscr_r1, gs))) return bail(st);
    if ((st = dalloc(p, &p->d_R1, (size_t)p->gmax * p->N)) || (st = dalloc(p, &p->d_r1view, nview)))
      return bail(st);
    std::vector<Rot1View> rv(nview);
    const double kHalfPi = 1.5707963267948966;
    const double rtol = 3.4526698300124393e-4;  // sqrt(eps(Float32)): isapprox default for a Float32 angle
    for (int v = 0; v < nview; ++v) {
      const double th = (double)p->angles[v];
      Rot1View r{0.0, 0.0, 0, 2};
      if (std::fmod(th, kTwoPi) == 0.0) {
        r.mode = 0;
      } else {
        long fl = (long)std::floor(0.5 + th / kHalfPi);
        r.m = (int)(((fl % 4) + 4) % 4);
        const double mh = r.m * kHalfPi;
        if (std::fabs(th - mh) <= rtol * std::max(std::fabs(th), std::fabs(mh))) {
          r.mode = 1;
        } else {
          const double mt = th - mh;
          r.tn = std::tan(mt / 2);
          r.sn = -std::sin(mt);
        }
      }
      rv[v] = r;
    }
    if ((st = up(p->d_r1view, rv.data(), sizeof(Rot1View) * nview))) return bail(st);
  }

  if (p->d_att && interpmeth == SPECT_INTERP_ONE) {
    // :one-rotated mu-map per group of views, then the depth scan
    cudaError_t e = cudaSuccess;
    for (int v0 = 0; v0 < nview && e == cudaSuccess; v0 += p->gmax) {
      const int nv = std::min(p->gmax, nview - v0);
      dim3 g1(nz, std::min(nv, p->r1_grid_y));
      k_rot1_fwd<<<g1, kRot1Threads, p->r1f_smem_ok ? p->r1f_smem : 0, hs>>>(
          p->r1, p->d_mumap, 0, p->d_r1view, p->d_all + v0, nv, p->d_R1, p->r1f_smem_ok, p->d_gscr_r1);
      const size_t n = (size_t)nv * nz * nx;
      k_att_scan<<<(int)std::min<size_t>((n + 255) / 256, (size_t)p->sm_count * 16), 256, 0, hs>>>(
          p->d_R1, nv, nx, ny, nz, dy, p->d_att + (size_t)v0 * p->N);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(hs);
    if (e != cudaSuccess) {
      fail(SPECT_ERR_CUDA, std::string("attenuation cache (:one): ") + cudaGetErrorString(e));
      return bail(SPECT_ERR_CUDA);
    }
  } else if (p->d_att && p->zpath) {
    // z-fastest cache from the mu-map laid out on the padded grid
    float* muz = nullptr;
    cudaError_t e = p->async_alloc ? cudaMallocAsync((void**)&muz, sizeof(float) * p->izN, hs)
                                   : cudaMalloc((void**)&muz, sizeof(float) * p->izN);
    if (e == cudaSuccess) e = cudaMemsetAsync(muz, 0, sizeof(float) * p->izN, hs);
    if (e == cudaSuccess) e = zto_iz_launch(p->zg, hs, p->d_mumap, muz);
    if (e == cudaSuccess) e = zatten_launch(p->zg, nview, hs, muz, p->d_rot, dy, p->d_att);
    if (e == cudaSuccess) e = cudaStreamSynchronize(hs);
    if (muz) dfree(p, muz);
    if (e != cudaSuccess) {
      fail(SPECT_ERR_CUDA, std::string("attenuation cache: ") + cudaGetErrorString(e));
      return bail(SPECT_ERR_CUDA);
    }
  } else if (p->d_att) {
    dim3 grid(nz, std::max(1, std::min(cdiv(2 * p->sm_count, nz), cdiv(nview, p->rotf_vpb))));
    const int thr = nx * p->rotf_vpb;
    if (p->att_smem_ok)
      k_atten_build<true><<<grid, thr, sizeof(float) * (size_t)nx * ny, hs>>>(g, p->d_mumap, p->d_rot, nview,
                                                                                p->d_att);
    else
      k_atten_build<false><<<grid, thr, 0, hs>>>(g, p->d_mumap, p->d_rot, nview, p->d_att);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(hs);
    if (e != cudaSuccess) {
      fail(SPECT_ERR_CUDA, std::string("attenuation cache: ") + cudaGetErrorString(e));
      return bail(SPECT_ERR_CUDA);
    }
  }

  // PSF spectra, in batches of planes (double precision on the device)
  {
    std::vector<double2> wx(Npx), wz(Npz);
    for (int m = 0; m < Npx; ++m) wx[m] = make_double2(std::cos(-kTwoPi * m / Npx), std::sin(-kTwoPi * m / Npx));
    for (int m = 0; m < Npz; ++m) wz[m] = make_double2(std::cos(-kTwoPi * m / Npz), std::sin(-kTwoPi * m / Npz));
    const size_t nplanes = (size_t)p->nset * ny;
    const size_t per_plane_G = (size_t)pz * Npx * sizeof(double2);
    const size_t batch = std::max<size_t>(1, std::min(nplanes, ((size_t)256 << 20) / per_plane_G));
    double2 *d_wx = nullptr, *d_wz = nullptr, *d_G = nullptr;
    float* d_psf = nullptr;
    float* d_Hfull = nullptr;
    auto tmalloc = [&](void** q, size_t b) {
      return p->async_alloc ? cudaMallocAsync(q, b, hs) : cudaMalloc(q, b);
    };
    auto cleanup = [&]() {
      dfree(p, d_wx);
      dfree(p, d_wz);
      dfree(p, d_G);
      dfree(p, d_psf);
      dfree(p, d_Hfull);
    };
    cudaError_t e = cudaSuccess;
    e = tmalloc((void**)&d_wx, sizeof(double2) * Npx);
    if (e == cudaSuccess) e = tmalloc((void**)&d_wz, sizeof(double2) * Npz);
    if (e == cudaSuccess) e = tmalloc((void**)&d_G, per_plane_G * batch);
    if (e == cudaSuccess) e = tmalloc((void**)&d_psf, sizeof(float) * pp * batch);
    if (e == cudaSuccess) e = tmalloc((void**)&d_Hfull, sizeof(float) * g.Hz * Npx * batch);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_wx, wx.data(), sizeof(double2) * Npx, cudaMemcpyHostToDevice, hs);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_wz, wz.data(), sizeof(double2) * Npz, cudaMemcpyHostToDevice, hs);
    std::vector<float> hp(pp * batch);
    for (size_t b0 = 0; e == cudaSuccess && b0 < nplanes; b0 += batch) {
      size_t nb = std::min(batch, nplanes - b0);
      if (opts.gauss) {  // planes b0.. of the single generated stack
        const int gb = std::min(cdiv((long long)nb * pp, 256), p->sm_count * 16);
        k_psf_gauss<<<gb, 256, 0, hs>>>(d_psf, (int)b0, (int)nb, ny, px, pz, opts.gx0, opts.gx1, opts.gz0, opts.gz1);
      } else {
        for (size_t q = 0; q < nb; ++q) {
          size_t pl = b0 + q;
          size_t set = pl / ny, y = pl % ny;
          std::memcpy(hp.data() + q * pp, psfs + ((size_t)uniq[set] * ny + y) * pp, sizeof(float) * pp);
        }
        e = cudaMemcpyAsync(d_psf, hp.data(), sizeof(float) * pp * nb, cudaMemcpyHostToDevice, hs);
      }
      if (e != cudaSuccess) break;
      int blocks = std::min(cdiv((long long)nb * pz * Npx, 256), p->sm_count * 32);
      k_psf_stage1<<<blocks, 256, 0, hs>>>(d_psf, (int)nb, px, pz, Npx, d_wx, d_G);
      blocks = std::min(cdiv((long long)nb * g.Hz * Npx, 256), p->sm_count * 32);
      k_psf_stage2<<<blocks, 256, 0, hs>>>(d_G, (int)nb, pz, Npx, Npz, g.Hz, d_wz, d_Hfull);
      const ConvGeom& cg = p->cg;
      blocks = std::min(cdiv((long long)nb * (cg.Q + 1) * Npx, 256), p->sm_count * 32);
      k_psf_permute<<<blocks, 256, 0, hs>>>(d_Hfull, (int)nb, Npx, Npz, g.Hz, p->RX, cg.logCX, p->RZ, cg.logCZ, cg.Q,
                                     p->d_H + b0 * (cg.Q + 1) * Npx);
      e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaStreamSynchronize(hs);
    }
    cleanup();
    if (e != cudaSuccess) {
      fail(SPECT_ERR_CUDA, std::string("PSF spectra: ") + cudaGetErrorString(e));
      return bail(SPECT_ERR_CUDA);
    }
  }
  // separable PSF planes: weight tables from the factors h = a b^T
  {
    const int zp = sep_zp(pz), xp = sep_xp(px), hs = zp + xp, hxs = (px - 1) / 2, hzs = (pz - 1) / 2;
    const int ts = std::max(4, (2 * hxs + 2 * hzs + 3) & ~3);
    std::vector<float> H((size_t)p->nset * ny * 2 * hs, 0.f), Tl((size_t)p->nset * ny * ts, 0.f);
    const bool ok = sep_host;
    std::vector<float> Hz, Ez;
    std::vector<int> Rz;
    std::vector<double> at(px), bt(pz);
    const char* trim_env = std::getenv("SPECT_ZTRIM");
    const bool trim = !(trim_env && trim_env[0] == '0');
    if (ok && p->zpath) {
      Hz.assign((size_t)p->nset * ny * 2 * zg.hs, 0.f);
      Ez.assign((size_t)p->nset * ny * 2 * zg.ts, 0.f);
      Rz.assign((size_t)p->nset * ny * 8, 0);
    }
    for (int u = 0; ok && u < p->nset; ++u)
      for (int y = 0; y < ny; ++y) {
        const double* a = fa.data() + ((size_t)u * ny + y) * px;
        const double* b = fb.data() + ((size_t)u * ny + y) * pz;
        // [wz reversed | wx reversed | b | a], each zero-padded (zp, xp)
        float* hrow = H.data() + ((size_t)u * ny + y) * 2 * hs;
        for (int m = 0; m < pz; ++m) hrow[m] = (float)b[pz - 1 - m];
        for (int m = 0; m < px; ++m) hrow[zp + m] = (float)a[px - 1 - m];
        for (int m = 0; m < pz; ++m) hrow[hs + m] = (float)b[m];
        for (int m = 0; m < px; ++m) hrow[hs + zp + m] = (float)a[m];
        // adjoint edge tails: cL_k = sum_{d>k} w(d), cR_k = sum_{d<-k} w(d)
        float* trow = Tl.data() + ((size_t)u * ny + y) * ts;
        fold_tails(a, hxs, trow, trow + hxs);
        fold_tails(b, hzs, trow + 2 * hxs, trow + 2 * hxs + hzs);
        if (!Hz.empty()) {
          // fused path, from the trimmed factors: [fwd z | fwd x | adj z |
          // adj x], each shifted right by its data offset minus the half
          // width; tails [ELz ERz ELx ERx | cLx cRx cLz cRz]; the tap-block
          // range of each pass
          std::copy(a, a + px, at.begin());
          std::copy(b, b + pz, bt.begin());
          if (trim) {
            trim_taps(at.data(), px);
            trim_taps(bt.data(), pz);
          }
          const int sz = zg.R0 - zg.hz, sx = zg.C0 - zg.hx;
          float* zr = Hz.data() + ((size_t)u * ny + y) * 2 * zg.hs;
          for (int m = 0; m < pz; ++m) zr[sz + m] = (float)bt[pz - 1 - m];
          for (int m = 0; m < px; ++m) zr[zg.zpw + sx + m] = (float)at[px - 1 - m];
          for (int m = 0; m < pz; ++m) zr[zg.hs + sz + m] = (float)bt[m];
          for (int m = 0; m < px; ++m) zr[zg.hs + zg.zpw + sx + m] = (float)at[m];
          float* er = Ez.data() + ((size_t)u * ny + y) * 2 * zg.ts;
          clamp_tails(bt.data(), pz, er, er + hzs);
          clamp_tails(at.data(), px, er + 2 * hzs, er + 2 * hzs + hxs);
          fold_tails(at.data(), hxs, er + zg.ts, er + zg.ts + hxs);
          fold_tails(bt.data(), hzs, er + zg.ts + 2 * hxs, er + zg.ts + 2 * hxs + hzs);
          for (int m = 0; m < pz; ++m) p->ztaps[0] += bt[m] != 0.0 ? 1.0 : 0.0;
          for (int m = 0; m < px; ++m) p->ztaps[1] += at[m] != 0.0 ? 1.0 : 0.0;
          int* rr = Rz.data() + ((size_t)u * ny + y) * 8;
          tap_range(zr, zg.zpw, rr, rr + 1);
          tap_range(zr + zg.zpw, zg.xpw, rr + 2, rr + 3);
          tap_range(zr + zg.hs, zg.zpw, rr + 4, rr + 5);
          tap_range(zr + zg.hs + zg.zpw, zg.xpw, rr + 6, rr + 7);
        }
      }
    if (!Hz.empty()) {
      p->ztaps[0] /= (double)p->nset * ny;
      p->ztaps[1] /= (double)p->nset * ny;
      if ((st = dalloc(p, &p->d_Hz, Hz.size())) || (st = up(p->d_Hz, Hz.data(), sizeof(float) * Hz.size())) ||
          (st = dalloc(p, &p->d_Ez, Ez.size())) || (st = up(p->d_Ez, Ez.data(), sizeof(float) * Ez.size())) ||
          (st = dalloc(p, &p->d_Rz, Rz.size())) || (st = up(p->d_Rz, Rz.data(), sizeof(int) * Rz.size())))
        return bail(st);
    }
    if (ok) {
      if ((st = dalloc(p, &p->d_Hsep, H.size())) || (st = up(p->d_Hsep, H.data(), sizeof(float) * H.size())) ||
          (st = dalloc(p, &p->d_Tsep, Tl.size())) || (st = up(p->d_Tsep, Tl.data(), sizeof(float) * Tl.size())))
        return bail(st);
      p->sep_ok = 1;
      p->sep_hs = hs;
      p->sep_ts = ts;
      const int att = (p->d_att && interpmeth == SPECT_INTERP_TWO) ? 1 : 0;
      p->sep_fwd_smem = sconv_fwd_smem(nx, nz, px, pz, att);
      // SPECT_CONV=fft: FFT kernels only; SPECT_CONV=direct: direct kernels
      // wherever they run (neither is then re-chosen by the autotuner)
      p->sep_forced = only_fft ? 1 : (conv_env && std::strcmp(conv_env, "direct") == 0) ? 2 : 0;
      p->sep_shape_fwd = nx % kSepXB == 0 ? sep_pick_shape(nx, nz, px, pz, true) : -1;
      p->sep_shape_adj = nx % kSepXB == 0 ? sep_pick_shape(nx, nz, px, pz, false) : -1;
      p->sep_fwd_ok = (p->sep_shape_fwd >= 0 && p->sep_fwd_smem <= p->max_smem) ? 1 : 0;
      p->sep = p->sep_fwd_ok && !only_fft;
      if (p->sep_fwd_ok)
        CUDA_TRY(cudaFuncSetAttribute(kSconvFwd[p->sep_shape_fwd], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)p->max_smem));
      // adjoint: multiplies the attenuation exactly when the rotation adjoint
      // expects premultiplied planes (adj_stage)
      p->sep_adj_smem = sconv_adj_smem(nx, nz, px, pz, ts, p->adj_stage ? 1 : 0);
      p->sep_adj_ok = (p->sep_shape_adj >= 0 && p->sep_adj_smem <= p->max_smem) ? 1 : 0;
      p->sep_adj = p->sep_adj_ok && !only_fft;
      if (p->sep_adj_ok)
        CUDA_TRY(cudaFuncSetAttribute(kSconvAdj[p->sep_shape_adj], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)p->max_smem));
    }
  }
  if (p->zpath) p->sep_fwd_ok = p->sep_adj_ok = p->sep = p->sep_adj = 1;  // direct convolution, fused
  *out = p;
  return SPECT_OK;
}
}  // namespace

extern "C" {

int spect_plan_create(spect_plan_t* out, int nx, int ny, int nz, int px, int pz, int nview, const float* mumap,
                      const float* psfs, float dy, const float* viewangle, int interpmeth, int mode, int nthread,
                      int nthreads) {
  return plan_create_impl(out, nx, ny, nz, px, pz, nview, mumap, psfs, dy, viewangle, interpmeth, mode, nthread,
                          nthreads, PlanOpts());
}

int spect_plan_destroy(spect_plan_t p) {
  if (!p) return fail(SPECT_ERR_ARG, "null plan");
  cudaDeviceSynchronize();
  free_plan(p);
  return SPECT_OK;
}

int spect_plan_info(spect_plan_t p, int out[8], size_t* bytes) {
  if (!p || !out) return fail(SPECT_ERR_ARG, "null pointer argument");
  int v[8] = {p->nx, p->ny, p->nz, p->px, p->pz, p->nview, p->interp, p->nset};
  std::memcpy(out, v, sizeof(v));
  if (bytes) *bytes = p->bytes;
  return SPECT_OK;
}

int spect_plan_conv_kernels(spect_plan_t p, int out[4]) {
  if (!p || !out) return fail(SPECT_ERR_ARG, "null pointer argument");
  std::lock_guard<std::mutex> lk(p->mu);
  out[0] = p->sep_fwd_ok;
  out[1] = p->sep_adj_ok;
  out[2] = p->sep;
  out[3] = p->sep_adj;
  return SPECT_OK;
}

int spect_plan_fused(spect_plan_t p, int* fused) {
  if (!p || !fused) return fail(SPECT_ERR_ARG, "null pointer argument");
  *fused = p->zpath;  // 1: fused pair; 2: large-plane kernels on the same layouts; 0: split kernels
  return SPECT_OK;
}

int spect_plan_fused_taps(spect_plan_t p, double* taps) {
  if (!p || !taps) return fail(SPECT_ERR_ARG, "null pointer argument");
  taps[0] = p->zpath ? p->ztaps[0] : (double)p->pz;
  taps[1] = p->zpath ? p->ztaps[1] : (double)p->px;
  return SPECT_OK;
}

int spect_project(spect_plan_t p, float* views, const float* image, const int32_t* index, int nindex, void* stream) {
  if (!p || !views || !image) return fail(SPECT_ERR_ARG, "null pointer argument");
  std::lock_guard<std::mutex> lk(p->mu);
  cudaStream_t st = (cudaStream_t)stream;
  const int* vi;
  STATUS_TRY(stage_index(p, index, nindex, st, &vi));
  return forward(p, views, image, vi, nindex, st, nullptr, nullptr);
}

int spect_project_static_scratch(spect_plan_t p, float* views, const float* image, const int32_t* index, int nindex,
                                 void* stream) {
  if (!p || !views || !image) return fail(SPECT_ERR_ARG, "null pointer argument");
  std::lock_guard<std::mutex> lk(p->mu);
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  if (dev != p->device)
    return fail(SPECT_ERR_ARG, "spect_project_static_scratch: the plan's device must be the current device");
  // views per group such that the rotated planes (N floats per view) and the
  // chunk partials (up to nchunk_max * nz * nx floats per view) fit
  const size_t per_view = sizeof(float) * (p->N + (size_t)p->nchunk_max * p->nxz) + 512;
  const size_t G = kStaticScratchBytes / per_view;
  if (G < 1)
    return fail(SPECT_ERR_UNSUPPORTED,
                "spect_project_static_scratch: one view needs " + std::to_string(per_view) +
                    " bytes of scratch, above the static limit of " + std::to_string(kStaticScratchBytes) + " bytes");
  void* base = nullptr;
  STATUS_TRY(static_scratch_address(&base));
  // groups never exceed the plan's own group size (the :one path stages
  // rotated slices in the plan buffer sized for p->gmax views)
  const int gmax = (int)std::min<size_t>(std::min<size_t>(G, (size_t)p->nview), (size_t)p->gmax);
  float* Pbuf = static_cast<float*>(base);
  size_t off = (sizeof(float) * (size_t)gmax * p->N + 255) & ~(size_t)255;
  float* partbuf = reinterpret_cast<float*>(static_cast<unsigned char*>(base) + off);
  cudaStream_t st = (cudaStream_t)stream;
  const int* vi;
  STATUS_TRY(stage_index(p, index, nindex, st, &vi));
  const bool prof = p->prof.on;
  p->prof.on = false;  // no event creation on this path
  int rc = forward_scratch(p, views, image, vi, nindex, st, nullptr, nullptr, Pbuf, partbuf, gmax);
  p->prof.on = prof;
  return rc;
}

// end of a host-synchronous call: wait for the stream, then report a kernel
// whose bounded wait on a bulk copy gave up (the flag is cleared)
int host_done(spect_plan_s* p, cudaStream_t st) {
  int h = 0;
  CUDA_TRY(cudaMemcpyAsync(&h, p->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  if (h) {
    CUDA_TRY(cudaMemset(p->d_err, 0, sizeof(int)));
    return fail(SPECT_ERR_TIMEOUT, "a bulk copy into shared memory did not complete");
  }
  return SPECT_OK;
}

int spect_project_host(spect_plan_t p, float* views, const float* image, const int32_t* index, int nindex) {
  if (!p || !views || !image) return fail(SPECT_ERR_ARG, "null pointer argument");
  std::lock_guard<std::mutex> lk(p->mu);
  STATUS_TRY(ensure_io(p));
  cudaStream_t st = 0;
  const int* vi;
  STATUS_TRY(stage_index(p, index, nindex, st, &vi));
  CUDA_TRY(cudaMemcpyAsync(p->d_io_img, image, sizeof(float) * p->N, cudaMemcpyHostToDevice, st));
  STATUS_TRY(forward(p, p->d_io_views, p->d_io_img, vi, nindex, st, nullptr, nullptr));
  CUDA_TRY(cudaMemcpyAsync(views, p->d_io_views, sizeof(float) * nindex * p->nxz, cudaMemcpyDeviceToHost, st));
  return host_done(p, st);
}

int spect_backproject(spect_plan_t p, float* image, const float* views, const int32_t* index, int nindex,
                      void* stream) {
  if (!p || !views || !image) return fail(SPECT_ERR_ARG, "null pointer argument");
  std::lock_guard<std::mutex> lk(p->mu);
  cudaStream_t st = (cudaStream_t)stream;
  const int* vi;
  STATUS_TRY(stage_index(p, index, nindex, st, &vi));
  return backward(p, image, views, vi, nindex, st, 0, nullptr);
}

int spect_backproject_host(spect_plan_t p, float* image, const float* views, const int32_t* index, int nindex) {
  if (!p || !views || !image) return fail(SPECT_ERR_ARG, "null pointer argument");
  std::lock_guard<std::mutex> lk(p->mu);
  STATUS_TRY(ensure_io(p));
  cudaStream_t st = 0;
  const int* vi;
  STATUS_TRY(stage_index(p, index, nindex, st, &vi));
  CUDA_TRY(cudaMemcpyAsync(p->d_io_views, views, sizeof(float) * nindex * p->nxz, cudaMemcpyHostToDevice, st));
  STATUS_TRY(backward(p, p->d_io_img, p->d_io_views, vi, nindex, st, 0, nullptr));
  CUDA_TRY(cudaMemcpyAsync(image, p->d_io_img, sizeof(float) * p->N, cudaMemcpyDeviceToHost, st));
  return host_done(p, st);
}

int spect_osem(spect_plan_t p, float* out, const float* x0, const float* ynoisy, const float* background, int nblocks,
               int niter, void* stream) {
  if (!p || !out || !x0 || !ynoisy || !background) return fail(SPECT_ERR_ARG, "null pointer argument");
  std::lock_guard<std::mutex> lk(p->mu);
  return run_osem(p, out, x0, ynoisy, background, nblocks, niter, (cudaStream_t)stream);
}

int spect_mlem(spect_plan_t p, float* out, const float* x0, const float* ynoisy, const float* background, int niter,
               void* stream) {
  return spect_osem(p, out, x0, ynoisy, background, 1, niter, stream);
}

int spect_osem_host(spect_plan_t p, float* out, const float* x0, const float* ynoisy, const float* background,
                    int nblocks, int niter) {
  if (!p || !out || !x0 || !ynoisy || !background) return fail(SPECT_ERR_ARG, "null pointer argument");
  std::lock_guard<std::mutex> lk(p->mu);
  size_t V = (size_t)p->nview * p->nxz;
  for (size_t k = 0; k < V; ++k)
    if (!(background[k] > 0.f)) return fail(SPECT_ERR_BACKGROUND, "need background > 0");
  STATUS_TRY(ensure_io(p));
  cudaStream_t st = 0;
  float* dx = p->d_io_img;
  float* dy = p->d_io_views;
  float* db = p->d_io_views + V;
  CUDA_TRY(cudaMemcpyAsync(dx, x0, sizeof(float) * p->N, cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(dy, ynoisy, sizeof(float) * V, cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(db, background, sizeof(float) * V, cudaMemcpyHostToDevice, st));
  STATUS_TRY(run_osem(p, dx, dx, dy, db, nblocks, niter, st));
  CUDA_TRY(cudaMemcpyAsync(out, dx, sizeof(float) * p->N, cudaMemcpyDeviceToHost, st));
  return host_done(p, st);
}

int spect_mlem_host(spect_plan_t p, float* out, const float* x0, const float* ynoisy, const float* background,
                    int niter) {
  return spect_osem_host(p, out, x0, ynoisy, background, 1, niter);
}

int spect_em_subset_update(spect_plan_t p, float* x, const float* ynoisy, const float* background, const float* asum,
                           const int32_t* index, int nindex, void* stream) {
  if (!p || !x || !ynoisy || !background || !asum) return fail(SPECT_ERR_ARG, "null pointer argument");
  std::lock_guard<std::mutex> lk(p->mu);
  cudaStream_t st = (cudaStream_t)stream;
  STATUS_TRY(ensure_em(p, 1));
  const int* vi;
  STATUS_TRY(stage_index(p, index, nindex, st, &vi));
  STATUS_TRY(forward(p, p->d_views_tmp, x, vi, nindex, st, ynoisy, background));
  return backward(p, x, p->d_views_tmp, vi, nindex, st, 2, asum);
}

int spect_subset_sensitivity(spect_plan_t p, float* asum, const int32_t* index, int nindex, void* stream) {
  if (!p || !asum) return fail(SPECT_ERR_ARG, "null pointer argument");
  std::lock_guard<std::mutex> lk(p->mu);
  cudaStream_t st = (cudaStream_t)stream;
  STATUS_TRY(ensure_em(p, 1));
  const int* vi;
  STATUS_TRY(stage_index(p, index, nindex, st, &vi));
  return backward(p, asum, p->d_ones, vi, nindex, st, 1, nullptr);
}

int spect_batch_create(spect_batch_t* out, int njobs, const spect_plan_t* plans, const int* nblocks,
                       const int* niter) {
  if (!out || !plans || !nblocks || !niter || njobs < 1) return fail(SPECT_ERR_ARG, "bad spect_batch_create arguments");
  *out = nullptr;
  for (int j = 0; j < njobs; ++j) {
    if (!plans[j]) return fail(SPECT_ERR_ARG, "null plan in batch");
    for (int k = 0; k < j; ++k)
      if (plans[k] == plans[j]) return fail(SPECT_ERR_ARG, "a plan may appear only once in a batch");
  }
  spect_batch_s* b = new spect_batch_s;
  auto bail = [&](int st) {
    spect_batch_destroy(b);
    return st;
  };
  b->plans.assign(plans, plans + njobs);
  b->nblocks.assign(nblocks, nblocks + njobs);
  b->niter.assign(niter, niter + njobs);
  b->out.assign(njobs, nullptr);
  b->x0.assign(njobs, nullptr);
  b->y.assign(njobs, nullptr);
  b->bg.assign(njobs, nullptr);
  for (int j = 0; j < njobs; ++j) {
    std::lock_guard<std::mutex> lk(b->plans[j]->mu);
    int st = prepare_osem(b->plans[j], nblocks[j], niter[j]);
    double f, a;
    if (st == SPECT_OK && (b->plans[j]->nview % nblocks[j]) == 0)
      st = autotune(b->plans[j], b->plans[j]->nview / nblocks[j], &f, &a);
    if (st != SPECT_OK) return bail(st);
  }
  if (cudaStreamCreateWithFlags(&b->root, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess)
    return bail(fail(SPECT_ERR_CUDA, "batch stream/event creation"));
  b->streams.assign(njobs, nullptr);
  b->done.assign(njobs, nullptr);
  for (int j = 0; j < njobs; ++j)
    if (cudaStreamCreateWithFlags(&b->streams[j], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->done[j], cudaEventDisableTiming) != cudaSuccess)
      return bail(fail(SPECT_ERR_CUDA, "batch stream/event creation"));
  *out = b;
  return SPECT_OK;
}

int spect_batch_set_job(spect_batch_t b, int job, float* out, const float* x0, const float* ynoisy,
                        const float* background) {
  if (!b || job < 0 || job >= (int)b->plans.size() || !out || !x0 || !ynoisy || !background)
    return fail(SPECT_ERR_ARG, "bad spect_batch_set_job arguments");
  std::lock_guard<std::mutex> lk(b->mu);
  spect_plan_s* p = b->plans[job];
  {
    std::lock_guard<std::mutex> lp(p->mu);
    STATUS_TRY(check_background(p, background, 0));
  }
  b->out[job] = out;
  b->x0[job] = x0;
  b->y[job] = ynoisy;
  b->bg[job] = background;
  b->dirty = true;
  return SPECT_OK;
}

int spect_batch_run(spect_batch_t b, void* stream) {
  if (!b) return fail(SPECT_ERR_ARG, "null batch");
  std::lock_guard<std::mutex> lk(b->mu);
  if (b->dirty) {
    std::vector<std::unique_lock<std::mutex>> locks;
    for (auto* p : b->plans) locks.emplace_back(p->mu);
    STATUS_TRY(batch_capture(b));
  }
  CUDA_TRY(cudaGraphLaunch(b->exec, (cudaStream_t)stream));
  g_launches.fetch_add(b->nkernels, std::memory_order_relaxed);
  return SPECT_OK;
}

int spect_batch_destroy(spect_batch_t b) {
  if (!b) return fail(SPECT_ERR_ARG, "null batch");
  cudaDeviceSynchronize();
  batch_release_graph(b);
  for (auto s : b->streams)
    if (s) cudaStreamDestroy(s);
  for (auto e : b->done)
    if (e) cudaEventDestroy(e);
  if (b->root) cudaStreamDestroy(b->root);
  if (b->fork) cudaEventDestroy(b->fork);
  delete b;
  return SPECT_OK;
}

int spect_plan_autotune(spect_plan_t p, int nindex, double ms[2]) {
  if (!p || nindex < 1 || nindex > p->nview) return fail(SPECT_ERR_ARG, "bad spect_plan_autotune arguments");
  std::lock_guard<std::mutex> lk(p->mu);
  double f = 0, a = 0;
  STATUS_TRY(autotune(p, nindex, &f, &a));
  if (ms) {
    ms[0] = f;
    ms[1] = a;
  }
  return SPECT_OK;
}

unsigned long long spect_kernel_launches(void) { return g_launches.load(); }

}  // extern "C"

namespace {
// the give-up path of the bounded mbarrier wait: a barrier that expects one
// arrival nobody makes (no copy is involved), a short bounded wait, the give-up
// recorded as the projector kernels' error exit does, and a normal return
__global__ void k_wait_giveup(int* err) {
  __shared__ unsigned long long bar;
  if (threadIdx.x == 0) mbar_init(&bar);
  __syncthreads();
  const bool ok = mbar_wait(&bar, 0u, 1 << 12);
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) atomicExch(err, 1);
    return;
  }
}

// independent FMA chains (x <- x a + b), 16 a thread: the FP32 pipe's rate
__global__ void __launch_bounds__(512) k_fma_chains(float* out, int iters, float a, float b) {
  float x[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) x[q] = threadIdx.x * 1e-3f + q;
  for (int i = 0; i < iters; ++i)
#pragma unroll
    for (int q = 0; q < 16; ++q) x[q] = fmaf(x[q], a, b);
  float s = 0.f;
#pragma unroll
  for (int q = 0; q < 16; ++q) s += x[q];
  if (s == 12345.f) out[0] = s;  // keeps the chains live
}
}  // namespace

extern "C" {

int spect_plan_check_error(spect_plan_t p, void* stream) {
  if (!p) return fail(SPECT_ERR_ARG, "null plan");
  std::lock_guard<std::mutex> lk(p->mu);
  int h = 0;
  cudaStream_t st = (cudaStream_t)stream;
  CUDA_TRY(cudaMemcpyAsync(&h, p->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  if (h) {
    CUDA_TRY(cudaMemsetAsync(p->d_err, 0, sizeof(int), st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return fail(SPECT_ERR_TIMEOUT, "a bulk copy into shared memory did not complete");
  }
  return SPECT_OK;
}

int spect_selftest_wait_timeout(void) {
  int* d = nullptr;
  CUDA_TRY(cudaMalloc(&d, sizeof(int)));
  cudaError_t e = cudaMemset(d, 0, sizeof(int));
  if (e == cudaSuccess) {
    k_wait_giveup<<<1, 32>>>(d);
    e = cudaGetLastError();
  }
  int h = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return fail(SPECT_ERR_CUDA, std::string("wait self-test: ") + cudaGetErrorString(e));
  if (h == 1) return fail(SPECT_ERR_TIMEOUT, "bounded wait gave up as intended (self-test)");
  return fail(SPECT_ERR_CUDA, "wait self-test: the bounded wait did not report its give-up");
}

int spect_fp32_peak(double* tflops) {
  if (!tflops) return fail(SPECT_ERR_ARG, "null pointer argument");
  int dev = 0, sms = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  float* d = nullptr;
  CUDA_TRY(cudaMalloc(&d, sizeof(float)));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int iters = 1 << 15, grid = 4 * sms, thr = 512;
  float best = 1e30f;
  cudaError_t e = cudaSuccess;
  for (int r = 0; r < 6 && e == cudaSuccess; ++r) {  // r = 0: warm-up
    cudaEventRecord(e0);
    k_fma_chains<<<grid, thr>>>(d, iters, 0.999f, 0.001f);
    cudaEventRecord(e1);
    e = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r > 0 && ms > 0.f) best = std::min(best, ms);
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  if (e != cudaSuccess) return fail(SPECT_ERR_CUDA, std::string("fp32 peak probe: ") + cudaGetErrorString(e));
  *tflops = (double)grid * thr * iters * 16 * 2 / (best * 1e-3) / 1e12;
  return SPECT_OK;
}

int spect_plan_profile(spect_plan_t p, int on) {
  if (!p) return fail(SPECT_ERR_ARG, "null plan");
  std::lock_guard<std::mutex> lk(p->mu);
  p->prof.reset();
  p->prof.on = on != 0;
  return SPECT_OK;
}

int spect_plan_kernel_times(spect_plan_t p, double ms[8], long long counts[8]) {
  if (!p || !ms || !counts) return fail(SPECT_ERR_ARG, "null pointer argument");
  std::lock_guard<std::mutex> lk(p->mu);
  p->prof.drain();
  for (int k = 0; k < K_KINDS; ++k) {
    ms[k] = p->prof.ms[k];
    counts[k] = p->prof.n[k];
  }
  return SPECT_OK;
}

int spect_psf_gauss(float* psf, int ny, int px, int pz, const double* fwhm_x, const double* fwhm_z) {
  if (!psf || !fwhm_x || ny <= 0 || px <= 0 || pz <= 0) return fail(SPECT_ERR_ARG, "bad psf_gauss arguments");
  if (!fwhm_z) fwhm_z = fwhm_x;
  auto gauss = [](int p, double fwhm, std::vector<double>& w) -> int {
    w.assign(p, 0.0);
    int h = (p - 1) / 2;
    if (fwhm == 0) {  // Kronecker impulse at r == 0
      bool has0 = false;
      for (int i = 0; i < p; ++i)
        if (-h + i == 0) {
          w[i] = 1.0;
          has0 = true;
        }
      return has0 ? 0 : -1;
    }
    double sigma = fwhm / std::sqrt(std::log(256.0));
    double s = 0;
    for (int i = 0; i < p; ++i) {
      double r = (double)(-h + i) / sigma;
      w[i] = std::exp(-0.5 * r * r);
      s += w[i];
    }
    for (auto& v : w) v /= s;
    return 0;
  };
  std::vector<double> wx, wz;
  for (int y = 0; y < ny; ++y) {
    if (gauss(px, fwhm_x[y], wx) || gauss(pz, fwhm_z[y], wz))
      return fail(SPECT_ERR_ARG, "must have some r=0 if fwhm=0");
    for (int j = 0; j < pz; ++j)
      for (int i = 0; i < px; ++i) psf[((size_t)y * pz + j) * px + i] = (float)(wx[i] * wz[j]);
  }
  return SPECT_OK;
}

int spect_psf_gauss_device(float* psf, int ny, int px, int pz, double fwhm_x_start, double fwhm_x_end,
                           double fwhm_z_start, double fwhm_z_end, void* stream) {
  if (!psf || ny <= 0 || px <= 0 || pz <= 0) return fail(SPECT_ERR_ARG, "bad psf_gauss arguments");
  if (!(px % 2) || !(pz % 2)) return fail(SPECT_ERR_PSF_NOT_ODD, "non-odd size psfs");
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  const long long n = (long long)ny * px * pz;
  k_psf_gauss<<<(int)std::min<long long>(cdiv(n, 256), (long long)sms * 16), 256, 0, (cudaStream_t)stream>>>(
      psf, 0, ny, ny, px, pz, fwhm_x_start, fwhm_x_end, fwhm_z_start, fwhm_z_end);
  return check_launch("k_psf_gauss");
}

int spect_plan_create_gauss(spect_plan_t* out, int nx, int ny, int nz, int px, int pz, int nview,
                            const float* mumap, double fwhm_x_start, double fwhm_x_end, double fwhm_z_start,
                            double fwhm_z_end, float dy, const float* viewangle, int interpmeth, int mode,
                            int nthread, int nthreads) {
  PlanOpts o;
  o.gauss = true;
  o.gx0 = fwhm_x_start;
  o.gx1 = fwhm_x_end;
  o.gz0 = fwhm_z_start;
  o.gz1 = fwhm_z_end;
  return plan_create_impl(out, nx, ny, nz, px, pz, nview, mumap, nullptr, dy, viewangle, interpmeth, mode, nthread,
                          nthreads, o);
}

}  // extern "C"

// ======================================================================
// Serving: continuous batching of OS-EM reconstruction requests.
// A scheduler thread admits pending jobs (FIFO) while a device-memory budget
// and a slot limit allow, builds each job's plan on the job's own
// non-blocking stream with stream-ordered allocation (no device-wide
// synchronisation, so admissions never stall running jobs), enqueues the
// whole osem! on that stream, and polls completion events; finished jobs
// release their memory and free slots for the next ones.  The jobs' work
// overlaps on the GPU.
namespace {

using Clock = std::chrono::steady_clock;

struct ServerJob {
  long long ticket = 0;
  int nx = 0, nz = 0, px = 0, pz = 0, nview = 0, interp = 2, nblocks = 1, niter = 1;
  float dy = 1.f;
  std::vector<float> mumap, psfs, y, bg, x0, result;  // psfs: the distinct stacks only
  std::vector<int> view_set;                          // view -> stack of psfs
  int state = 0;  // 0 pending, 1 active, 2 done, 3 failed
  int status = SPECT_OK;
  std::string err;
  Clock::time_point t_submit, t_admit, t_done;
  size_t est = 0, bytes = 0;
  spect_plan_s* plan = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t ev = nullptr;
  float *d_x = nullptr, *d_x0 = nullptr, *d_y = nullptr, *d_bg = nullptr;
  float* h_out = nullptr;  // pinned result (from the server's pool), filled on the job's stream
  size_t h_cap = 0;
};

size_t est_job_bytes(const ServerJob& j, bool att) {
  const size_t N = (size_t)j.nx * j.nx * j.nz, nxz = (size_t)j.nx * j.nz;
  const int Npx = power2(j.nx + j.px - 1), Npz = power2(j.nz + j.pz - 1);
  const size_t Q = std::max(1, Npz / 2), nsub = j.nview / j.nblocks;
  size_t f = N                                       // mumap
             + (att ? (size_t)j.nview * N : 0)        // attenuation cache
             + (size_t)j.nx * (Q + 1) * Npx           // PSF spectra (one set)
             + nsub * N + nsub * 16 * nxz + 2 * nsub * Q * Npx  // P, part, Vs
             + 8 * N + 2 * (size_t)j.nview * nxz + (size_t)j.nblocks * N  // imgpart, EM buffers
             + 2 * N + 2 * (size_t)j.nview * nxz;     // job buffers
  if (j.interp == SPECT_INTERP_ONE) f += nsub * N;
  else f += 2 * nsub * (size_t)j.nx * j.nx * ((j.nz + 15) / 16 * 16) + 2 * N;  // z-fastest planes and tiles, IZ volumes
  size_t b = 4 * f + (size_t)j.nview * 32;
  // per-CTA global slabs of large planes (B, spectra accumulators)
  if ((size_t)j.nx * (Q + 1) * 8 + 8192 > 227 * 1024) b += (size_t)148 * j.nx * (Q + 1) * 8;
  if ((Npx / std::min(32, Npx)) * (Npz / std::min(32, Npz)) > 32) b += (size_t)148 * Q * Npx * 8;
  const size_t slice = (size_t)j.nx * j.nx;
  if ((2 * slice + 4 * (size_t)j.nx) * 4 > 227 * 1024) b += (size_t)j.nz * 8 * (2 * slice + 512) * 4;
  if (j.nx * 32 * nxz * 4 > ((size_t)256 << 20)) b += 0;  // part stays at 16 chunks
  return b + b / 10 + ((size_t)16 << 20);
}

}  // namespace

constexpr int kServerThreads = 4;

struct spect_server_s {
  size_t budget = 0;
  int max_active = 1;
  int device = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<ServerJob*> pending;
  std::vector<ServerJob*> active;
  std::unordered_map<long long, ServerJob*> jobs;
  long long next_ticket = 1;
  size_t used = 0;
  bool stop = false;
  long long n_submitted = 0, n_done = 0, n_failed = 0, max_active_seen = 0;
  // scheduler threads: each admits and retires jobs; while one prepares a
  // job's plan on the host (validation, uploads, PSF spectra) the others
  // keep admitting and retiring
  std::vector<std::thread> workers;
  // pinned result buffers, reused across jobs (freed at destroy: freeing
  // pinned memory synchronises the device)
  std::mutex pool_mu;
  std::vector<std::pair<float*, size_t>> pool;
};

namespace {

// pinned buffer of at least n floats from the pool (or a new one)
float* pool_get(spect_server_s* S, size_t n, size_t* cap) {
  {
    std::lock_guard<std::mutex> lk(S->pool_mu);
    for (size_t i = 0; i < S->pool.size(); ++i)
      if (S->pool[i].second >= n) {
        float* q = S->pool[i].first;
        *cap = S->pool[i].second;
        S->pool.erase(S->pool.begin() + i);
        return q;
      }
  }
  float* q = nullptr;
  if (cudaMallocHost((void**)&q, sizeof(float) * n) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  *cap = n;
  return q;
}

void pool_put(spect_server_s* S, float* q, size_t cap) {
  if (!q) return;
  std::lock_guard<std::mutex> lk(S->pool_mu);
  S->pool.push_back({q, cap});
}

// releases a finished job's device resources (stream-ordered frees on its
// stream; the stream is destroyed once its queued work has run) and returns
// its pinned buffer to the pool; no device-wide synchronisation
void job_release(spect_server_s* S, ServerJob* j) {
  if (j->plan) free_plan(j->plan);  // stream-ordered frees on the job's stream
  j->plan = nullptr;
  float* bufs[] = {j->d_x, j->d_x0, j->d_y, j->d_bg};
  for (float* q : bufs)
    if (q) cudaFreeAsync(q, j->st);
  j->d_x = j->d_x0 = j->d_y = j->d_bg = nullptr;
  if (j->ev) cudaEventDestroy(j->ev);
  if (j->st) cudaStreamDestroy(j->st);  // released once its queued frees ran
  j->ev = nullptr;
  j->st = nullptr;
  pool_put(S, j->h_out, j->h_cap);
  j->h_out = nullptr;
  j->h_cap = 0;
  std::vector<float>().swap(j->mumap);
  std::vector<float>().swap(j->psfs);
  std::vector<float>().swap(j->y);
  std::vector<float>().swap(j->bg);
  std::vector<float>().swap(j->x0);
}

int job_admit(spect_server_s* S, ServerJob* j, size_t budget) {
  CUDA_TRY(cudaStreamCreateWithFlags(&j->st, cudaStreamNonBlocking));
  CUDA_TRY(cudaEventCreateWithFlags(&j->ev, cudaEventDisableTiming));
  PlanOpts o;
  o.home = j->st;
  o.async_alloc = true;
  o.gmax_cap = j->nview / j->nblocks;
  const size_t att = sizeof(float) * (size_t)j->nx * j->nx * j->nz * j->nview;
  o.atten_cache = (j->interp == SPECT_INTERP_ONE || att <= budget / 8) ? 1 : 0;
  o.view_set = j->view_set.data();
  o.nset = (int)(j->psfs.size() / ((size_t)j->nx * j->px * j->pz));
  spect_plan_t plan = nullptr;
  STATUS_TRY(plan_create_impl(&plan, j->nx, j->nx, j->nz, j->px, j->pz, j->nview, j->mumap.data(), j->psfs.data(),
                              j->dy, nullptr, j->interp, SPECT_MODE_FAST, 1, 1, o));
  j->plan = plan;
  const size_t N = plan->N, V = (size_t)j->nview * plan->nxz;
  STATUS_TRY(dalloc(plan, &j->d_x, N));
  STATUS_TRY(dalloc(plan, &j->d_x0, N));
  STATUS_TRY(dalloc(plan, &j->d_y, V));
  STATUS_TRY(dalloc(plan, &j->d_bg, V));
  // the plan frees what dalloc took; keep job buffers out of its list
  CUDA_TRY(cudaMemcpyAsync(j->d_x0, j->x0.data(), sizeof(float) * N, cudaMemcpyHostToDevice, j->st));
  CUDA_TRY(cudaMemcpyAsync(j->d_y, j->y.data(), sizeof(float) * V, cudaMemcpyHostToDevice, j->st));
  CUDA_TRY(cudaMemcpyAsync(j->d_bg, j->bg.data(), sizeof(float) * V, cudaMemcpyHostToDevice, j->st));
  STATUS_TRY(prepare_osem(plan, j->nblocks, j->niter));
  STATUS_TRY(enqueue_osem(plan, j->d_x, j->d_x0, j->d_y, j->d_bg, j->nblocks, j->niter, j->st));
  // the result lands in pinned memory before the completion event
  j->h_out = pool_get(S, N, &j->h_cap);
  if (!j->h_out) return fail(SPECT_ERR_OOM, "pinned result buffer");
  CUDA_TRY(cudaMemcpyAsync(j->h_out, j->d_x, sizeof(float) * N, cudaMemcpyDeviceToHost, j->st));
  CUDA_TRY(cudaEventRecord(j->ev, j->st));
  j->bytes = std::max(plan->bytes, j->est);  // conservative accounting
  return SPECT_OK;
}

void server_loop(spect_server_s* S) {
  cudaSetDevice(S->device);
  std::unique_lock<std::mutex> lk(S->mu);
  std::vector<std::pair<ServerJob*, cudaError_t>> finished;
  for (;;) {
    // completions: poll the events (non-blocking) under the lock, then copy
    // the pinned results and release the jobs outside it
    finished.clear();
    for (size_t i = 0; i < S->active.size();) {
      ServerJob* j = S->active[i];
      const cudaError_t q = cudaEventQuery(j->ev);
      if (q == cudaErrorNotReady) {
        ++i;
        continue;
      }
      finished.push_back({j, q});
      S->used -= std::min(S->used, j->bytes);
      S->active.erase(S->active.begin() + i);
    }
    if (!finished.empty()) {
      lk.unlock();
      for (auto& f : finished) {
        ServerJob* j = f.first;
        if (f.second == cudaSuccess) j->result.assign(j->h_out, j->h_out + j->plan->N);
        j->t_done = Clock::now();
        job_release(S, j);
      }
      lk.lock();
      for (auto& f : finished) {
        ServerJob* j = f.first;
        if (f.second == cudaSuccess) {
          j->state = 2;
          S->n_done++;
        } else {
          j->state = 3;
          j->status = SPECT_ERR_CUDA;
          j->err = std::string("job execution: ") + cudaGetErrorString(f.second);
          S->n_failed++;
        }
      }
      S->cv_done.notify_all();
    }
    // admissions (FIFO) while slots and memory allow
    while (!S->pending.empty() && (int)S->active.size() < S->max_active && !S->stop) {
      ServerJob* j = S->pending.front();
      if (j->est > S->budget) {
        S->pending.pop_front();
        j->state = 3;
        j->status = SPECT_ERR_OOM;
        j->err = "job needs about " + std::to_string(j->est) + " bytes, above the server budget of " +
                 std::to_string(S->budget);
        j->t_done = Clock::now();
        S->n_failed++;
        S->cv_done.notify_all();
        continue;
      }
      if (S->used + j->est > S->budget) break;  // wait for memory to free up
      S->pending.pop_front();
      S->used += j->est;
      lk.unlock();
      j->t_admit = Clock::now();
      const int rc = job_admit(S, j, S->budget);
      std::string err = rc == SPECT_OK ? std::string() : g_err;
      if (rc != SPECT_OK) {
        j->t_done = Clock::now();
        job_release(S, j);
      }
      lk.lock();
      S->used -= j->est;
      if (rc != SPECT_OK) {
        j->state = 3;
        j->status = rc;
        j->err = err;
        S->n_failed++;
        S->cv_done.notify_all();
        continue;
      }
      S->used += j->bytes;
      j->state = 1;
      S->active.push_back(j);
      S->max_active_seen = std::max<long long>(S->max_active_seen, (long long)S->active.size());
    }
    if (S->stop && S->active.empty()) break;
    if (S->active.empty() && S->pending.empty()) {
      S->cv_work.wait(lk, [&] { return S->stop || !S->pending.empty(); });
    } else {
      lk.unlock();
      std::this_thread::sleep_for(std::chrono::microseconds(50));
      lk.lock();
    }
  }
}

}  // namespace

extern "C" {

int spect_server_create(spect_server_t* out, size_t device_budget, int max_active) {
  if (!out || max_active < 1) return fail(SPECT_ERR_ARG, "bad spect_server_create arguments");
  *out = nullptr;
  spect_server_s* S = new spect_server_s;
  if (cudaGetDevice(&S->device) != cudaSuccess) {
    delete S;
    return fail(SPECT_ERR_CUDA, "no CUDA device");
  }
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) fr = 0;
  S->budget = device_budget ? device_budget : fr / 2;
  S->max_active = max_active;
  for (int t = 0; t < kServerThreads; ++t) S->workers.emplace_back(server_loop, S);
  *out = S;
  return SPECT_OK;
}

int spect_server_submit(spect_server_t S, const spect_job_desc* d, long long* ticket) {
  if (!S || !d || !ticket || !d->mumap || !d->psfs || !d->ynoisy || !d->background)
    return fail(SPECT_ERR_ARG, "bad spect_server_submit arguments");
  if (d->nx <= 0 || d->nz <= 0 || d->px <= 0 || d->pz <= 0 || d->nview <= 0)
    return fail(SPECT_ERR_ARG, "sizes must be positive");
  if ((d->nx % 2)) return fail(SPECT_ERR_NX_ODD, "nx odd");
  if (!(d->px % 2) || !(d->pz % 2)) return fail(SPECT_ERR_PSF_NOT_ODD, "non-odd size psfs");
  if (d->interpmeth != SPECT_INTERP_ONE && d->interpmeth != SPECT_INTERP_TWO)
    return fail(SPECT_ERR_INTERP, "bad interpmeth");
  if (d->nblocks < 1 || d->nview % d->nblocks != 0) return fail(SPECT_ERR_NBLOCKS, "nview must be divisible by nblocks!");
  if (d->niter < 0) return fail(SPECT_ERR_ARG, "niter must be >= 0");
  const size_t N = (size_t)d->nx * d->nx * d->nz, V = (size_t)d->nx * d->nz * d->nview;
  for (size_t k = 0; k < V; ++k)
    if (!(d->background[k] > 0.f)) return fail(SPECT_ERR_BACKGROUND, "need background > 0");
  const size_t pp = (size_t)d->px * d->pz, stack = (size_t)d->nx * pp;
  std::vector<int> view_set, uniq;
  psf_sets(d->psfs, d->nview, stack, view_set, uniq);
  if (!psf_symmetric(d->psfs, uniq, d->nx, pp)) return fail(SPECT_ERR_PSF_ASYM, "asym. psf");
  if (power2(d->nx + d->px - 1) > SPECT_TW_N || power2(d->nz + d->pz - 1) > SPECT_TW_N)
    return fail(SPECT_ERR_UNSUPPORTED, "padded plane exceeds this build's FFT limit");
  ServerJob* j = new ServerJob;
  j->nx = d->nx;
  j->nz = d->nz;
  j->px = d->px;
  j->pz = d->pz;
  j->nview = d->nview;
  j->interp = d->interpmeth;
  j->nblocks = d->nblocks;
  j->niter = d->niter;
  j->dy = d->dy;
  j->mumap.assign(d->mumap, d->mumap + N);
  j->psfs.resize(uniq.size() * stack);
  for (size_t u = 0; u < uniq.size(); ++u)
    std::memcpy(j->psfs.data() + u * stack, d->psfs + (size_t)uniq[u] * stack, sizeof(float) * stack);
  j->view_set = std::move(view_set);
  j->y.assign(d->ynoisy, d->ynoisy + V);
  j->bg.assign(d->background, d->background + V);
  if (d->x0) j->x0.assign(d->x0, d->x0 + N);
  else j->x0.assign(N, 1.0f);
  j->est = est_job_bytes(*j, j->interp == SPECT_INTERP_ONE ||
                                 sizeof(float) * N * j->nview <= S->budget / 8);
  j->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) {
      delete j;
      return fail(SPECT_ERR_BUSY, "server is shutting down");
    }
    j->ticket = S->next_ticket++;
    S->jobs[j->ticket] = j;
    S->pending.push_back(j);
    S->n_submitted++;
  }
  S->cv_work.notify_one();
  *ticket = j->ticket;
  return SPECT_OK;
}

int spect_server_wait(spect_server_t S, long long ticket, float* out, double* latency_ms, int timeout_ms) {
  if (!S) return fail(SPECT_ERR_ARG, "null server");
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->jobs.find(ticket);
  if (it == S->jobs.end()) return fail(SPECT_ERR_ARG, "unknown ticket " + std::to_string(ticket));
  ServerJob* j = it->second;
  auto done = [&] { return j->state >= 2; };
  if (timeout_ms < 0) S->cv_done.wait(lk, done);
  else if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done))
    return fail(SPECT_ERR_TIMEOUT, "job " + std::to_string(ticket) + " not finished");
  S->jobs.erase(it);
  lk.unlock();
  if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(j->t_done - j->t_submit).count();
  int rc = j->status;
  if (rc == SPECT_OK && out) std::memcpy(out, j->result.data(), sizeof(float) * j->result.size());
  if (rc != SPECT_OK) g_err = j->err;
  delete j;
  return rc;
}

int spect_server_stats(spect_server_t S, long long out[8]) {
  if (!S || !out) return fail(SPECT_ERR_ARG, "null pointer argument");
  std::lock_guard<std::mutex> lk(S->mu);
  long long v[8] = {S->n_submitted, S->n_done, S->n_failed, (long long)S->active.size(),
                    (long long)S->pending.size(), S->max_active_seen, (long long)S->used, (long long)S->budget};
  std::memcpy(out, v, sizeof(v));
  return SPECT_OK;
}

int spect_server_destroy(spect_server_t S) {
  if (!S) return fail(SPECT_ERR_ARG, "null server");
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
    for (ServerJob* j : S->pending) {
      j->state = 3;
      j->status = SPECT_ERR_BUSY;
      j->err = "server shut down before the job was admitted";
    }
    S->pending.clear();
  }
  S->cv_work.notify_all();
  for (auto& w : S->workers)
    if (w.joinable()) w.join();  // running jobs finish first
  for (auto& kv : S->jobs) delete kv.second;
  for (auto& b : S->pool) cudaFreeHost(b.first);
  delete S;
  return SPECT_OK;
}

}  // extern "C"
