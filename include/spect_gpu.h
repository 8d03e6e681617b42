/* spect_gpu.h -- C ABI of libspectgpu.so, the B200 (sm_100a) SPECT projector.
 *
 * Drop-in boundary for the hot path of SPECTrecon.jl: the bodies of
 * SPECTplan / project! / backproject! / mlem! / osem! become calls into this
 * library (Julia `ccall`, Python `ctypes`).  Plain pointers and sizes only.
 *
 * Array layout is the reference's Julia column-major layout, unchanged:
 *   image [nx,ny,nz]        -> C row-major float[nz][ny][nx]
 *   mumap [nx,ny,nz]        -> float[nz][ny][nx]
 *   views [nx,nz,nview]     -> float[nview][nz][nx]
 *   psfs  [px,pz,ny,nview]  -> float[nview][ny][pz][px]
 * View indices are 0-based here (the Julia shim subtracts 1).
 *
 * Every entry point returns an int status (SPECT_OK == 0); the message of the
 * last failure on the calling thread is spect_last_error().  The messages of
 * the reference's own throws are kept verbatim (see the status list).
 *
 * Pointer kinds: functions named *_host take host arrays and are synchronous
 * (they copy in, compute, copy out).  The others take device pointers and
 * enqueue on `stream` (a cudaStream_t, NULL = legacy default stream); they
 * return as soon as the work is queued.
 *
 * Threading: calls on one plan are serialised on the plan's work buffers, so
 * use one plan per host thread (the reference plan is not re-entrant either,
 * src/spectplan.jl:95-112).  Distinct plans may run concurrently.
 */
#ifndef SPECT_GPU_H
#define SPECT_GPU_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes; messages mirror the reference's throws */
enum {
  SPECT_OK = 0,
  SPECT_ERR_NX_NE_NY = 1,      /* "nx != ny"            src/spectplan.jl:76 */
  SPECT_ERR_NX_ODD = 2,        /* "nx odd"              src/spectplan.jl:77 */
  SPECT_ERR_PSF_NOT_ODD = 3,   /* "non-odd size psfs"   src/spectplan.jl:82 */
  SPECT_ERR_PSF_ASYM = 4,      /* "asym. psf"           src/spectplan.jl:83-84 */
  SPECT_ERR_INTERP = 5,        /* "bad interpmeth"      src/spectplan.jl:87 */
  SPECT_ERR_NTHREAD = 6,       /* "bad nthread"         src/spectplan.jl:90 */
  SPECT_ERR_MODE = 7,          /* "bad mode"            src/spectplan.jl:93 */
  SPECT_ERR_DIM = 8,           /* DimensionMismatch     src/project.jl:204-205, src/ml-os-em.jl:25-26 */
  SPECT_ERR_BACKGROUND = 9,    /* "need background > 0" src/ml-os-em.jl:30,106 */
  SPECT_ERR_NBLOCKS = 10,      /* "nview must be divisible by nblocks!" src/ml-os-em.jl:73 */
  SPECT_ERR_INDEX = 11,        /* view index out of 0..nview-1 (Julia BoundsError) */
  SPECT_ERR_ARG = 12,          /* null pointer / non-positive size */
  SPECT_ERR_UNSUPPORTED = 13,  /* size beyond this build's kernel limits */
  SPECT_ERR_CUDA = 14,         /* CUDA runtime error (message has the detail) */
  SPECT_ERR_OOM = 15,          /* device allocation failed / memory budget */
  SPECT_ERR_TIMEOUT = 16,      /* a bounded device wait gave up */
  SPECT_ERR_BUSY = 17          /* resource in use (serving slot table full) */
};

/* interpolation method of SPECTplan(...; interpmeth) */
enum { SPECT_INTERP_ONE = 1, SPECT_INTERP_TWO = 2 };
/* SPECTplan(...; mode): accepted and validated, no effect on the GPU */
enum { SPECT_MODE_FAST = 0, SPECT_MODE_MEM = 1 };

typedef struct spect_plan_s* spect_plan_t;

/* Message of the last failing call on this thread ("" if none). */
const char* spect_last_error(void);

/* Library/device information: fills sm count, total device memory (bytes). */
int spect_device_info(int* sm_count, size_t* total_mem);

/* SPECTplan(mumap, psfs, dy; T, viewangle, interpmeth, nthread, mode)
 * (src/spectplan.jl:58-137).  mumap and psfs are HOST arrays;
 * they are validated exactly as the reference does (nx == ny, nx even, px/pz
 * odd, every psfs[:,:,y,v] point-symmetric, interpmeth, nthread == nthreads,
 * mode), uploaded, and the PSF spectra are precomputed on the device.  Unlike
 * the reference plan, later edits of the host mumap/psfs are not seen.
 * viewangle may be NULL for the default (0:nview-1)/nview*2pi rounded to
 * Float32; otherwise nview angles in radians.  `nthreads` is the caller's
 * thread count (Julia: Threads.nthreads()). */
int spect_plan_create(spect_plan_t* plan, int nx, int ny, int nz, int px, int pz, int nview,
                      const float* mumap, const float* psfs, float dy, const float* viewangle,
                      int interpmeth, int mode, int nthread, int nthreads);
int spect_plan_destroy(spect_plan_t plan);

/* Sizes and device memory held by the plan: out[0..7] = nx, ny, nz, px, pz,
 * nview, interpmeth, number of distinct PSF spectrum sets; *bytes = device
 * bytes held by the plan. */
int spect_plan_info(spect_plan_t plan, int out[8], size_t* bytes);

/* Convolution kernels of the plan (no reference counterpart: the reference
 * always convolves by FFT, src/fft_convolve.jl:33-130).  out[0], out[1]: the
 * direct separable kernels can run for the forward / adjoint (every PSF plane
 * is rank-1); out[2], out[3]: the forward / adjoint currently uses them
 * (1) or the FFT kernels (0).  spect_plan_autotune keeps the faster. */
int spect_plan_conv_kernels(spect_plan_t plan, int out[4]);

/* 1 in *fused when the plan runs the fused projector pair (rotation,
 * attenuation, separable PSF convolution and depth sum in one forward kernel;
 * the adjoint convolution then an atomic-free gather rotation adjoint with
 * the EM update fused); 2 when it runs the large-plane kernels (the same
 * layouts and passes, one kernel per pass over plane tiles: planes too large
 * for the fused kernels' shared memory; SPECT_ZSTRIP=1 prefers them, =0 never
 * takes them); 0 when it runs the split kernels.  1 and 2 are used for :two
 * plans with the attenuation cache and rank-1 PSF planes of at most 69 taps
 * (SPECT_ZPATH=0 turns both off).  No counterpart in the reference (query of
 * this implementation's kernel choice). */
int spect_plan_fused(spect_plan_t plan, int* fused);

/* taps[0], taps[1]: mean number of PSF taps per depth plane that the plan's
 * z and x convolution passes run.  The fused pair skips the outer taps of
 * each plane's factors whose summed magnitude per side is within 2^-27 of the
 * factor's (below Float32 resolution; SPECT_ZTRIM=0 keeps them); other plans
 * report pz and px.  No counterpart in the reference (work accounting of this
 * implementation). */
int spect_plan_fused_taps(spect_plan_t plan, double* taps);

/* project!(views, image, plan; index) (src/project.jl:143-163).
 * views[nindex][nz][nx] = P_{index[i]} image; index NULL = all views in order
 * (nindex must then be nview).  Device pointers, enqueued on stream. */
int spect_project(spect_plan_t plan, float* views, const float* image, const int32_t* index, int nindex,
                  void* stream);
/* Same with host arrays; synchronous. */
int spect_project_host(spect_plan_t plan, float* views, const float* image, const int32_t* index,
                       int nindex);

/* Forward projection that allocates nothing (no counterpart in the
 * reference).  Same result as spect_project, for callers that cannot call
 * cudaMalloc once their plan exists: processes whose device memory is
 * reserved up front by another allocator (a serving framework's memory
 * pool), and real-time acquisition pipelines that forbid allocation after
 * start-up.  Its scratch (the rotated planes and the depth-chunk partial
 * views) lives in one file-scope device array of 32 MiB that every GPU
 * loading this library holds until the process exits; the views are
 * processed in groups that fit it, and a plan whose single view needs more
 * (nx*ny*nz + 32*nx*nz floats > 32 MiB) is rejected with
 * SPECT_ERR_UNSUPPORTED.  The first call on a device looks up the array's
 * device address (cudaGetSymbolAddress); make that first call before any
 * stream capture.  All calls share the array and no part of it needs to
 * start at zero, but calls that overlap on the GPU (other streams, other
 * threads) race on it: serialise them.  Device pointers, enqueued on
 * stream; the plan's device must be the current device.  The array's device
 * address is looked up once per device and kept for the life of the process,
 * so resetting a device (cudaDeviceReset) while the library is loaded is not
 * supported by this entry point. */
int spect_project_static_scratch(spect_plan_t plan, float* views, const float* image, const int32_t* index,
                                 int nindex, void* stream);

/* backproject!(image, views, plan; index) (src/backproject.jl:132-162).  image = sum_i P_{index[i]}' views[i]; image need not be zeroed. */
int spect_backproject(spect_plan_t plan, float* image, const float* views, const int32_t* index,
                      int nindex, void* stream);
int spect_backproject_host(spect_plan_t plan, float* image, const float* views, const int32_t* index,
                           int nindex);

/* mlem!(out, x0, ynoisy, background, A; niter) (src/ml-os-em.jl:21-49) with A the plan's full projector.  Device pointers; the
 * EM ratio is fused into the forward reduction and the multiplicative update
 * into the back-projection's last stage. */
int spect_mlem(spect_plan_t plan, float* out, const float* x0, const float* ynoisy,
               const float* background, int niter, void* stream);
int spect_mlem_host(spect_plan_t plan, float* out, const float* x0, const float* ynoisy,
                    const float* background, int niter);

/* osem!(out, x0, ynoisy, background, Ablock(plan, nblocks); niter)
 * (src/ml-os-em.jl:70-131): subsets nb:nblocks:nview. */
int spect_osem(spect_plan_t plan, float* out, const float* x0, const float* ynoisy,
               const float* background, int nblocks, int niter, void* stream);
int spect_osem_host(spect_plan_t plan, float* out, const float* x0, const float* ynoisy,
                    const float* background, int nblocks, int niter);

/* One fused OS-EM subset update on device buffers (the loop body of
 * src/ml-os-em.jl:120-127):
 *   x .*= A_s' (y_s ./ (A_s x + b_s)) ./ asum
 * y and background are the FULL [nview][nz][nx] arrays; the subset is
 * index[0..nindex).  asum is A_s' 1 with zeros replaced by +Inf. */
int spect_em_subset_update(spect_plan_t plan, float* x, const float* ynoisy, const float* background,
                           const float* asum, const int32_t* index, int nindex, void* stream);

/* asum = A_s' 1 with zeros replaced by +Inf (src/ml-os-em.jl:111-114). */
int spect_subset_sensitivity(spect_plan_t plan, float* asum, const int32_t* index, int nindex,
                             void* stream);

/* Autotuner (no counterpart in the reference).  Times candidate launch
 * shapes of the plan's forward and adjoint projector for nindex views on the
 * device (the depth-chunk tile of the FFT-convolution kernels, the view split
 * of the rotation kernels) and keeps the fastest for calls with nindex views;
 * results are cached per plan shape in the process.  ms[0], ms[1]: best
 * forward and adjoint times.  Synchronous; spect_batch_create runs it for
 * every job's subset size. */
int spect_plan_autotune(spect_plan_t plan, int nindex, double ms[2]);

/* Batched OS-EM (no counterpart in the reference: its osem! runs one
 * reconstruction at a time).  A batch holds njobs plans of any sizes (each
 * plan at most once) with their subset counts and iteration counts.  Every
 * job's whole osem! (sensitivities, then niter x nblocks fused subset
 * updates) is enqueued on its own stream and captured once into a single
 * CUDA graph; spect_batch_run launches that graph on `stream` (one launch
 * for all reconstructions; the jobs overlap on the GPU).  set_job gives the
 * device buffers of job j (out, x0 [nz][ny][nx]; ynoisy, background
 * [nview][nz][nx]) and checks background > 0 (synchronously); changing a
 * job's buffers re-captures the graph at the next run. */
typedef struct spect_batch_s* spect_batch_t;
int spect_batch_create(spect_batch_t* batch, int njobs, const spect_plan_t* plans, const int* nblocks,
                       const int* niter);
int spect_batch_set_job(spect_batch_t batch, int job, float* out, const float* x0, const float* ynoisy,
                        const float* background);
int spect_batch_run(spect_batch_t batch, void* stream);
int spect_batch_destroy(spect_batch_t batch);

/* Serving (no counterpart in the reference).  A server runs OS-EM
 * reconstruction requests with continuous batching: a scheduler thread
 * admits pending requests in arrival order while the device-memory budget
 * (0 = half of the free memory) and max_active slots allow, keeps each
 * admitted job's plan, PSF spectra, attenuation and iterate resident on the
 * GPU, runs it on its own stream (jobs of different sizes overlap on the
 * device), and frees its memory when it finishes so waiting requests can be
 * admitted.  submit validates like SPECTplan/osem! (same messages), copies the
 * host arrays and returns at once; wait blocks until the job is done (or
 * timeout_ms, < 0 = forever), copies the reconstruction [nz][ny][nx] to `out`
 * and the submit-to-finish latency to latency_ms.  stats: submitted, done,
 * failed, active, pending, most active at once, bytes in use, budget. */
typedef struct {
  int nx, nz, px, pz, nview;     /* ny = nx */
  const float* mumap;            /* [nz][ny][nx] */
  const float* psfs;             /* [nview][ny][pz][px] */
  float dy;
  int interpmeth;                /* SPECT_INTERP_ONE / SPECT_INTERP_TWO */
  const float* ynoisy;           /* [nview][nz][nx] */
  const float* background;       /* [nview][nz][nx], > 0 */
  const float* x0;               /* [nz][ny][nx] or NULL (ones) */
  int nblocks, niter;
} spect_job_desc;
typedef struct spect_server_s* spect_server_t;
int spect_server_create(spect_server_t* server, size_t device_budget, int max_active);
int spect_server_submit(spect_server_t server, const spect_job_desc* job, long long* ticket);
int spect_server_wait(spect_server_t server, long long ticket, float* out, double* latency_ms, int timeout_ms);
int spect_server_stats(spect_server_t server, long long out[8]);
int spect_server_destroy(spect_server_t server);

/* Kernel accounting (no counterpart in the reference; measurement support).
 * spect_kernel_launches: number of kernels this library has launched in the
 * process.  spect_plan_profile(plan, on): when on, every kernel the plan
 * launches is bracketed by CUDA events on its stream; spect_plan_kernel_times
 * synchronises on those events and returns, per kernel kind, the summed
 * device milliseconds and launch counts since profiling was switched on:
 * index 0 k_rot_fwd, 1 k_conv_fwd, 2 k_reduce_views, 3 k_vspec,
 * 4 k_conv_adj, 5 k_rot_adj, 6 k_reduce_image, 7 other. */
unsigned long long spect_kernel_launches(void);

/* Failure detection of the bounded device waits (no counterpart in the
 * reference).  Every kernel that waits for a bulk copy into shared memory
 * polls its mbarrier a bounded number of times; on give-up it sets the plan's
 * error flag and returns, so the context stays usable.  The *_host entry
 * points report the flag as SPECT_ERR_TIMEOUT; callers of the asynchronous
 * (device-pointer) entry points read and clear it with
 * spect_plan_check_error(plan), which synchronises the plan's flag read on
 * `stream` and returns SPECT_OK or SPECT_ERR_TIMEOUT.
 * spect_selftest_wait_timeout() exercises the give-up path on the current
 * device: one block waits a short bounded time on an mbarrier whose single
 * expected arrival never happens, records the give-up and returns; the call returns
 * SPECT_ERR_TIMEOUT when that path worked (and SPECT_ERR_CUDA if the kernel
 * failed).  Synchronous; allocates 4 bytes. */
int spect_plan_check_error(spect_plan_t plan, void* stream);
int spect_selftest_wait_timeout(void);
int spect_plan_profile(spect_plan_t plan, int on);
int spect_plan_kernel_times(spect_plan_t plan, double ms[8], long long counts[8]);

/* FP32 (CUDA-core) peak of the current device, measured: independent FFMA
 * chains on every SM (4 blocks x 512 threads per SM, 16 chains a thread),
 * best of 5 timed launches; writes TFLOP/s (2 FLOP per FMA).  The roofline
 * denominator for this path's FP32-bound kernels (no counterpart in the
 * reference; measurement support).  Synchronous. */
int spect_fp32_peak(double* tflops);

/* psf_gauss(; ny, px, pz, fwhm_x, fwhm_z) (src/psf-gauss.jl:24-55): host
 * generator of depth-dependent Gaussian PSFs into psf[ny][pz][px] (Julia
 * psf[px,pz,ny]).  fwhm_x/fwhm_z hold ny values (fwhm_z NULL = fwhm_x). */
int spect_psf_gauss(float* psf, int ny, int px, int pz, const double* fwhm_x, const double* fwhm_z);

/* psf_gauss on the device (src/psf-gauss.jl:24-55, with fwhm = range(start,
 * end, ny) per axis): writes psf[ny][pz][px] (device memory of the caller)
 * on `stream`, in double precision rounded to float like spect_psf_gauss. */
int spect_psf_gauss_device(float* psf, int ny, int px, int pz, double fwhm_x_start, double fwhm_x_end,
                           double fwhm_z_start, double fwhm_z_end, void* stream);

/* SPECTplan with the Gaussian PSF stack psf_gauss(; ny, px, pz, fwhm ranges)
 * for every view (the repeated-PSF use of docs/lit/examples/1-overview.jl:
 * 91-104), generated on the device: no host PSF array, one stack of PSF
 * spectra.  Otherwise as spect_plan_create. */
int spect_plan_create_gauss(spect_plan_t* plan, int nx, int ny, int nz, int px, int pz, int nview,
                            const float* mumap, double fwhm_x_start, double fwhm_x_end, double fwhm_z_start,
                            double fwhm_z_end, float dy, const float* viewangle, int interpmeth, int mode,
                            int nthread, int nthreads);

#ifdef __cplusplus
}
#endif

#endif /* SPECT_GPU_H */
