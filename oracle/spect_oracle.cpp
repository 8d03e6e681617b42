// spect_oracle.cpp -- CPU ORACLE (test infrastructure only).
//
// This file is the checker for the CUDA projector, not part of the product.
// Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
// arm may load liboracle.so.  It restates, in plain C++17, the algorithm of
// SPECTrecon.jl's SPECT projector hot path, function by function, in both
// float (the reference's Float32 run) and double (the Float64 run used for
// error statements):
//
//   Power2/_padup/_paddown/_padleft/_padright   src/helper.jl:8-12
//   padzero!, padrepl!, pad2sizezero!            src/helper.jl:20-80
//   fftshift2!                                   src/helper.jl:111-142
//   imfilterz!, fft_conv!, fft_conv_adj!         src/fft_convolve.jl:16-130
//   linearinterp!, rotate_x!/_y!(_adj)           src/rotatez.jl:21-147
//   rotl90!, rotr90!, rot180!, rot_f90!(_adj)    src/rotatez.jl:155-230
//   imrotate!/imrotate_adj! (:one)               src/rotatez.jl:240-322
//   imrotate!/imrotate_adj! (:two)               src/rotatez.jl:331-416
//   project! (per view, multi-view :fast)        src/project.jl:77-163
//   backproject! (per view, multi-view :fast)    src/backproject.jl:69-162
//   spawner                                      src/spawn.jl:10-17
//   mlem!, osem!, Ablock subsets                 src/ml-os-em.jl:21-131
//   viewangle default                            src/spectplan.jl:63
//   PlanRotate padsize                           src/plan-rotate.jl:56
//
// Third-party arithmetic restated from its published definition:
//   * FFTW (FFTW.jl, compat "1"): unnormalised forward DFT with exp(-2*pi*i*k*n/N),
//     inverse scaled by 1/N (AbstractFFTs ScaledPlan).  Restated here as a
//     radix-2 decimation-in-time FFT; rounding therefore differs from FFTW at
//     the 1e-7 level, never in value.
//   * LinearInterpolators.jl (compat "0.1"): SparseInterpolator y[i] = sum of its
//     two (coefficient, index) pairs, adjoint = the transposed scatter;
//     TwoDimensionalTransformInterpolator with LinearSpline = bilinear sampling
//     of the zero-padded input at R(u) = c + Rot(2*pi - theta)(u - c).  All
//     samples of the cropped centre fall inside the padded grid, so the
//     kernel's boundary mode never changes a value.
//
// Parity status: the reference is Julia and no Julia runs on these machines,
// so no output of the reference itself pins this restatement.  It is pinned by
// the reference's own known-answer tests (test/helper.jl, test/rotatez.jl,
// test/psf-gauss.jl), its adjoint tests (test/adjoint-*.jl, test/fftconv.jl),
// the FFT-convolution == replicate-boundary direct convolution identity, and
// the agreement of the :one (fully specified in the reference source) and :two
// rotations.  The 2-D bilinear values of LinearInterpolators are pinned only
// indirectly, through that :one/:two agreement.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

constexpr double kTwoPi = 6.283185307179586;  // Julia's 2pi as Float64
constexpr double kHalfPi = 1.5707963267948966;

inline int power2(int x) {  // Power2 = x -> 2^(ceil(Int, log2(x)))
  int p = 1;
  while (p < x) p <<= 1;
  return p;
}
inline int ceil_half(int a) { return (a + 1) / 2; }  // ceil(a/2), a >= 0
inline int floor_half(int a) { return a / 2; }
inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// spawner(fun!, nthread, ntask): contiguous chunks of ceil(ntask/nthread)
// tasks, chunk k handled by buffer k (src/spawn.jl:10-17).
template <class F>
void spawner(int nthread, int ntask, F&& fun) {
  if (ntask <= 0) return;
  int chunk = (ntask + nthread - 1) / nthread;
  std::vector<std::thread> th;
  int buffer = 0;
  for (int start = 0; start < ntask; start += chunk, ++buffer) {
    int stop = std::min(ntask, start + chunk);
    th.emplace_back([=, &fun]() {
      for (int t = start; t < stop; ++t) fun(buffer, t);
    });
  }
  for (auto& t : th) t.join();
}

// ---------------------------------------------------------------- FFT ----
template <class T>
struct FFT1 {
  int n = 0, logn = 0;
  std::vector<int> rev;
  std::vector<T> wr, wi;  // exp(-2 pi i k / n), k < n/2
  explicit FFT1(int n_) : n(n_) {
    while ((1 << logn) < n) ++logn;
    rev.resize(n);
    for (int i = 0; i < n; ++i) {
      int r = 0;
      for (int b = 0; b < logn; ++b)
        if (i & (1 << b)) r |= 1 << (logn - 1 - b);
      rev[i] = r;
    }
    wr.resize(std::max(1, n / 2));
    wi.resize(std::max(1, n / 2));
    for (int k = 0; k < n / 2; ++k) {
      double a = -kTwoPi * k / n;
      wr[k] = (T)std::cos(a);
      wi[k] = (T)std::sin(a);
    }
  }
  // in-place complex DFT of n contiguous (re,im) pairs; inverse is unscaled
  void run(T* re, T* im, bool inverse) const {
    for (int i = 0; i < n; ++i) {
      int r = rev[i];
      if (r > i) {
        std::swap(re[i], re[r]);
        std::swap(im[i], im[r]);
      }
    }
    for (int len = 2; len <= n; len <<= 1) {
      int half = len / 2, step = n / len;
      for (int s = 0; s < n; s += len) {
        for (int k = 0; k < half; ++k) {
          T c = wr[k * step], d = inverse ? -wi[k * step] : wi[k * step];
          int a = s + k, b = a + half;
          T xr = re[b] * c - im[b] * d;
          T xi = re[b] * d + im[b] * c;
          re[b] = re[a] - xr;
          im[b] = im[a] - xi;
          re[a] = re[a] + xr;
          im[a] = im[a] + xi;
        }
      }
    }
  }
};

// The DFT of FFT1 applied to every line along dim 2 of an m x n column-major
// split array (line i = entries i, i + m, ...), all m lines at once: the same
// bit reversal, butterflies and twiddles as FFT1::run, so each line's result
// is bit-identical to FFT1::run on that line; the inner loop runs over the
// contiguous dim 1 (vectorisable, unit stride).
template <class T>
void dft_along2(T* re, T* im, int m, const FFT1<T>& f, bool inverse) {
  const int n = f.n;
  for (int j = 0; j < n; ++j) {
    const int r = f.rev[j];
    if (r > j) {
      std::swap_ranges(re + (size_t)j * m, re + (size_t)(j + 1) * m, re + (size_t)r * m);
      std::swap_ranges(im + (size_t)j * m, im + (size_t)(j + 1) * m, im + (size_t)r * m);
    }
  }
  for (int len = 2; len <= n; len <<= 1) {
    const int half = len / 2, step = n / len;
    for (int s = 0; s < n; s += len)
      for (int k = 0; k < half; ++k) {
        const T c = f.wr[k * step], d = inverse ? -f.wi[k * step] : f.wi[k * step];
        T* __restrict ra = re + (size_t)(s + k) * m;
        T* __restrict ia = im + (size_t)(s + k) * m;
        T* __restrict rb = re + (size_t)(s + k + half) * m;
        T* __restrict ib = im + (size_t)(s + k + half) * m;
        for (int i = 0; i < m; ++i) {
          const T xr = rb[i] * c - ib[i] * d;
          const T xi = rb[i] * d + ib[i] * c;
          rb[i] = ra[i] - xr;
          ib[i] = ia[i] - xi;
          ra[i] = ra[i] + xr;
          ia[i] = ia[i] + xi;
        }
      }
  }
}

// dst (n2 x n1) = transpose of src (n1 x n2), column-major, in cache tiles
template <class T>
void transpose_cm(T* __restrict dst, const T* __restrict src, int n1, int n2) {
  constexpr int B = 16;
  for (int j0 = 0; j0 < n2; j0 += B)
    for (int i0 = 0; i0 < n1; i0 += B)
      for (int j = j0; j < std::min(n2, j0 + B); ++j)
        for (int i = i0; i < std::min(n1, i0 + B); ++i) dst[j + (size_t)i * n2] = src[i + (size_t)j * n1];
}

// 2-D DFT of an n1 x n2 column-major complex array (split re/im): the 1-D
// DFT along dim 1 of every column, then along dim 2 of every row (each line
// exactly FFT1::run).  Dim 1 runs on a transposed copy so that both passes
// sweep contiguous memory.
template <class T>
struct FFT2 {
  int n1, n2;
  FFT1<T> f1, f2;
  std::vector<T> tr, ti;
  FFT2(int a, int b) : n1(a), n2(b), f1(a), f2(b), tr((size_t)a * b), ti((size_t)a * b) {}
  void run(T* re, T* im, bool inverse) {
    transpose_cm(tr.data(), re, n1, n2);
    transpose_cm(ti.data(), im, n1, n2);
    dft_along2(tr.data(), ti.data(), n2, f1, inverse);
    transpose_cm(re, tr.data(), n2, n1);
    transpose_cm(im, ti.data(), n2, n1);
    dft_along2(re, im, n1, f2, inverse);
    if (inverse) {  // AbstractFFTs ScaledPlan: multiply by 1/N
      T s = (T)(1.0 / ((double)n1 * n2));
      size_t N = (size_t)n1 * n2;
      for (size_t k = 0; k < N; ++k) {
        re[k] *= s;
        im[k] *= s;
      }
    }
  }
};

// --------------------------------------------------------- PlanPSF -------
// Work buffers of one PlanPSF (src/plan-psf.jl:26-109).
template <class T>
struct PsfWork {
  int nx, nz, px, pz, Npx, Npz, padup, paddown, padleft, padright;
  FFT2<T> fft;
  std::vector<T> ir, ii, kr, ki, work, vecx, vecz;
  PsfWork(int nx_, int nz_, int px_, int pz_)
      : nx(nx_), nz(nz_), px(px_), pz(pz_), Npx(power2(nx_ + px_ - 1)), Npz(power2(nz_ + pz_ - 1)),
        padup(ceil_half(Npx - nx_)), paddown(floor_half(Npx - nx_)),
        padleft(ceil_half(Npz - nz_)), padright(floor_half(Npz - nz_)), fft(Npx, Npz) {
    size_t N = (size_t)Npx * Npz;
    ir.resize(N); ii.resize(N); kr.resize(N); ki.resize(N); work.resize(N);
    vecx.resize(Npx); vecz.resize(Npz);
  }
  // pad2sizezero!(ker_compl, ker, size) (src/helper.jl:66-80)
  void load_kernel(const T* ker) {
    std::fill(kr.begin(), kr.end(), T(0));
    std::fill(ki.begin(), ki.end(), T(0));
    int pd1 = ceil_half(Npx - px), pd2 = ceil_half(Npz - pz);
    for (int j = 0; j < pz; ++j)
      for (int i = 0; i < px; ++i) kr[(pd1 + i) + (size_t)(pd2 + j) * Npx] = ker[i + (size_t)j * px];
  }
  // imfilterz! (src/fft_convolve.jl:16-25): FFT, multiply, IFFT, fftshift2!,
  // real part into work.
  void imfilterz() {
    fft.run(ir.data(), ii.data(), false);
    fft.run(kr.data(), ki.data(), false);
    size_t N = (size_t)Npx * Npz;
    for (size_t k = 0; k < N; ++k) {
      T a = ir[k], b = ii[k], c = kr[k], d = ki[k];
      ir[k] = a * c - b * d;
      ii[k] = a * d + b * c;
    }
    fft.run(ir.data(), ii.data(), true);
    int m = Npx / 2, n = Npz / 2;  // fftshift2!: dst[i,j] = src[(i+m)%Npx, (j+n)%Npz]
    for (int j = 0; j < Npz; ++j) {
      const T* src = ir.data() + (size_t)((j + n) % Npz) * Npx;
      T* dst = work.data() + (size_t)j * Npx;
      for (int i = 0; i < Npx - m; ++i) dst[i] = src[i + m];
      for (int i = Npx - m; i < Npx; ++i) dst[i] = src[i + m - Npx];
    }
  }
};

// fft_conv!(output, img, ker, plan) (src/fft_convolve.jl:33-55)
template <class T>
void fft_conv(T* out, const T* img, const T* ker, PsfWork<T>& w, size_t ostride_z, size_t istride_z) {
  const int nx = w.nx, nz = w.nz, Npx = w.Npx, Npz = w.Npz;
  for (int j = 0; j < Npz; ++j) {  // padrepl!
    int jz = clampi(j - w.padleft, 0, nz - 1);
    for (int i = 0; i < Npx; ++i) {
      int ix = clampi(i - w.padup, 0, nx - 1);
      w.ir[i + (size_t)j * Npx] = img[ix + jz * istride_z];
      w.ii[i + (size_t)j * Npx] = T(0);
    }
  }
  w.load_kernel(ker);
  w.imfilterz();
  for (int j = 0; j < nz; ++j)
    for (int i = 0; i < nx; ++i) out[i + j * ostride_z] = w.work[(w.padup + i) + (size_t)(w.padleft + j) * Npx];
}

// fft_conv_adj!(output, img, ker, plan) (src/fft_convolve.jl:82-130)
template <class T>
void fft_conv_adj(T* out, const T* img, const T* ker, PsfWork<T>& w, size_t ostride_z, size_t istride_z) {
  const int nx = w.nx, nz = w.nz, Npx = w.Npx, Npz = w.Npz;
  std::fill(w.ir.begin(), w.ir.end(), T(0));  // padzero!
  std::fill(w.ii.begin(), w.ii.end(), T(0));
  for (int j = 0; j < nz; ++j)
    for (int i = 0; i < nx; ++i) w.ir[(w.padup + i) + (size_t)(w.padleft + j) * Npx] = img[i + j * istride_z];
  w.load_kernel(ker);
  w.imfilterz();
  T* W = w.work.data();
  // adjoint of replicate padding: rows then columns
  std::fill(w.vecz.begin(), w.vecz.end(), T(0));
  for (int i = 0; i < w.padup; ++i)
    for (int m = 0; m < Npz; ++m) w.vecz[m] += W[i + (size_t)m * Npx];
  for (int m = 0; m < Npz; ++m) W[w.padup + (size_t)m * Npx] += w.vecz[m];
  std::fill(w.vecz.begin(), w.vecz.end(), T(0));
  for (int i = w.padup + nx; i < Npx; ++i)
    for (int m = 0; m < Npz; ++m) w.vecz[m] += W[i + (size_t)m * Npx];
  for (int m = 0; m < Npz; ++m) W[(w.padup + nx - 1) + (size_t)m * Npx] += w.vecz[m];
  std::fill(w.vecx.begin(), w.vecx.end(), T(0));
  for (int j = 0; j < w.padleft; ++j)
    for (int n = 0; n < Npx; ++n) w.vecx[n] += W[n + (size_t)j * Npx];
  for (int n = 0; n < Npx; ++n) W[n + (size_t)w.padleft * Npx] += w.vecx[n];
  std::fill(w.vecx.begin(), w.vecx.end(), T(0));
  for (int j = w.padleft + nz; j < Npz; ++j)
    for (int n = 0; n < Npx; ++n) w.vecx[n] += W[n + (size_t)j * Npx];
  for (int n = 0; n < Npx; ++n) W[n + (size_t)(w.padleft + nz - 1) * Npx] += w.vecx[n];
  for (int j = 0; j < nz; ++j)
    for (int i = 0; i < nx; ++i) out[i + j * ostride_z] = W[(w.padup + i) + (size_t)(w.padleft + j) * Npx];
}

// ------------------------------------------------------- rotation --------
inline int rot_padsize(int nx) {  // ceil(Int, 1 + nx*sqrt(2)/2 - nx/2)
  return (int)std::ceil(1.0 + nx * std::sqrt(2.0) / 2.0 - nx / 2.0);
}

template <class T>
struct RotWork {
  int nx, pad, L;
  std::vector<T> w1, w2;
  std::vector<T> C;    // SparseInterpolator coefficients (2 per row)
  std::vector<int> J;  // 1-based indices
  explicit RotWork(int nx_) : nx(nx_), pad(rot_padsize(nx_)), L(nx_ + 2 * rot_padsize(nx_)) {
    w1.resize((size_t)L * L);
    w2.resize((size_t)L * L);
    C.resize(2 * L);
    J.resize(2 * L);
  }
  // padzero!(work, img, (pad,pad,pad,pad))
  void padzero(std::vector<T>& dst, const T* img, size_t istride) const {
    std::fill(dst.begin(), dst.end(), T(0));
    for (int j = 0; j < nx; ++j)
      for (int i = 0; i < nx; ++i) dst[(pad + i) + (size_t)(pad + j) * L] = img[i + j * istride];
  }
  void crop(T* out, const std::vector<T>& src, size_t ostride) const {
    for (int j = 0; j < nx; ++j)
      for (int i = 0; i < nx; ++i) out[i + j * ostride] = src[(pad + i) + (size_t)(pad + j) * L];
  }
  // linearinterp!(A, s, e, len) (src/rotatez.jl:21-51): s, e in Float64,
  // coefficients rounded to T when stored.
  void linearinterp(double s, double e, int len) {
    double dec = std::ceil(s) - s;
    int ncoeff = 2 * len, ncol = len;
    for (int i = 1; i <= ncoeff; ++i) C[i - 1] = (i & 1) ? (T)dec : (T)(1.0 - dec);
    if (e <= ncol) {
      J[ncoeff - 1] = (int)std::ceil(e);
      for (int i = ncoeff - 1; i >= 1; --i) J[i - 1] = std::max(1, J[ncoeff - 1] - (ncoeff - i + 1) / 2);
    } else {
      J[0] = (int)std::floor(s);
      for (int i = 2; i <= ncoeff; ++i) J[i - 1] = std::min(ncol, J[0] + i / 2);
    }
  }
  // y = A x along a strided line (SparseInterpolator mul!)
  void apply(T* y, const T* x, size_t stride) const {
    for (int r = 0; r < L; ++r) {
      T s = T(0);
      s += C[2 * r] * x[(size_t)(J[2 * r] - 1) * stride];
      s += C[2 * r + 1] * x[(size_t)(J[2 * r + 1] - 1) * stride];
      y[(size_t)r * stride] = s;
    }
  }
  // y = A' x (transposed scatter)
  void apply_adj(T* y, const T* x, size_t stride) const {
    for (int r = 0; r < L; ++r) y[(size_t)r * stride] = T(0);
    for (int r = 0; r < L; ++r) {
      T a = x[(size_t)r * stride];
      y[(size_t)(J[2 * r] - 1) * stride] += C[2 * r] * a;
      y[(size_t)(J[2 * r + 1] - 1) * stride] += C[2 * r + 1] * a;
    }
  }
  // rotate_x!/rotate_x_adj! (src/rotatez.jl:57-99): lines along dim 1
  void rotate_x(std::vector<T>& out, const std::vector<T>& img, double tan_t, bool adj) {
    double c = (L + 1) / 2.0;
    for (int i = 1; i <= L; ++i) {
      double s = (i - c) * tan_t + 1, e = (i - c) * tan_t + L;
      linearinterp(s, e, L);
      if (adj) apply_adj(out.data() + (size_t)(i - 1) * L, img.data() + (size_t)(i - 1) * L, 1);
      else apply(out.data() + (size_t)(i - 1) * L, img.data() + (size_t)(i - 1) * L, 1);
    }
  }
  // rotate_y!/rotate_y_adj! (src/rotatez.jl:105-147): lines along dim 2
  void rotate_y(std::vector<T>& out, const std::vector<T>& img, double sin_t, bool adj) {
    double c = (L + 1) / 2.0;
    for (int i = 1; i <= L; ++i) {
      double s = (i - c) * sin_t + 1, e = (i - c) * sin_t + L;
      linearinterp(s, e, L);
      if (adj) apply_adj(out.data() + (i - 1), img.data() + (i - 1), L);
      else apply(out.data() + (i - 1), img.data() + (i - 1), L);
    }
  }
};

// rotl90!, rotr90!, rot180! on L x L column-major (src/rotatez.jl:155-190)
template <class T>
void rotl90(T* B, const T* A, int L) {
  for (int i = 0; i < L; ++i)
    for (int j = 0; j < L; ++j) B[(L - 1 - j) + (size_t)i * L] = A[i + (size_t)j * L];
}
template <class T>
void rotr90(T* B, const T* A, int L) {
  for (int i = 0; i < L; ++i)
    for (int j = 0; j < L; ++j) B[j + (size_t)(L - 1 - i) * L] = A[i + (size_t)j * L];
}
template <class T>
void rot180(T* B, const T* A, int L) {
  for (int j = 0; j < L; ++j)
    for (int i = 0; i < L; ++i) B[(L - 1 - i) + (size_t)(L - 1 - j) * L] = A[i + (size_t)j * L];
}
// rot_f90!/rot_f90_adj! (src/rotatez.jl:197-230); returns -1 for bad m
template <class T>
int rot_f90(T* out, const T* img, int L, int m, bool adj) {
  if (m == 0) std::memcpy(out, img, sizeof(T) * (size_t)L * L);
  else if (m == 1) (adj ? rotr90<T> : rotl90<T>)(out, img, L);
  else if (m == 2) rot180<T>(out, img, L);
  else if (m == 3) (adj ? rotl90<T> : rotr90<T>)(out, img, L);
  else return -1;
  return 0;
}

template <class T> constexpr double rtol_default();
template <> constexpr double rtol_default<float>() { return 3.4526698300124393e-4; }   // sqrt(eps(Float32))
template <> constexpr double rtol_default<double>() { return 1.4901161193847656e-8; }  // sqrt(eps(Float64))

// imrotate!/imrotate_adj! with :one (src/rotatez.jl:240-322).  theta has the
// plan's element type; the shear parameters are Float64 as in the reference.
template <class T>
void imrotate_one(T* out, const T* img, T theta_t, RotWork<T>& w, bool adj, size_t stride) {
  const int nx = w.nx, L = w.L;
  double theta = (double)theta_t;
  if (std::fmod(theta, kTwoPi) == 0.0) {  // mod(theta, 2pi) ≈ 0 holds only at exactly 0
    for (int j = 0; j < nx; ++j)
      for (int i = 0; i < nx; ++i) out[i + j * stride] = img[i + j * stride];
    return;
  }
  long fl = (long)std::floor(0.5 + theta / kHalfPi);
  int m = (int)(((fl % 4) + 4) % 4);
  double mh = m * kHalfPi;
  bool near90 = std::fabs(theta - mh) <= rtol_default<T>() * std::max(std::fabs(theta), std::fabs(mh));
  if (near90) {
    w.padzero(w.w2, img, stride);
    rot_f90(w.w1.data(), w.w2.data(), L, m, adj);
  } else {
    double mt = theta - mh;
    double tn = std::tan(mt / 2), sn = -std::sin(mt);
    w.padzero(w.w1, img, stride);
    if (!adj) {
      rot_f90(w.w2.data(), w.w1.data(), L, m, false);
      w.rotate_x(w.w1, w.w2, tn, false);
      w.rotate_y(w.w2, w.w1, sn, false);
      w.rotate_x(w.w1, w.w2, tn, false);
    } else {
      w.rotate_x(w.w2, w.w1, tn, true);
      w.rotate_y(w.w1, w.w2, sn, true);
      w.rotate_x(w.w2, w.w1, tn, true);
      rot_f90(w.w1.data(), w.w2.data(), L, m, true);
    }
  }
  w.crop(out, w.w1, stride);
}

// :two bilinear sampling coefficients for angle theta.  The reference builds
// c + rotate(2pi - theta, AffineTransform2D{T}() - c); 2pi - theta is Float64,
// its cos/sin are stored in T.  Output pixel (i,j) (0-based, unpadded) samples
// the input at s = c0 + Rot(phi) (o - c0), c0 = (nx-1)/2, Rot(phi) =
// [cos -sin; sin cos] acting on (dim1, dim2).
template <class T>
struct Rot2 {
  T cs, sn, c0;
  Rot2(T theta, int nx) {
    double phi = kTwoPi - (double)theta;
    cs = (T)std::cos(phi);
    sn = (T)std::sin(phi);
    c0 = (T)((nx - 1) * 0.5);
  }
  // sample position of output pixel (i, j); same operation order as the GPU
  inline void pos(int i, int j, T& s1, T& s2) const {
    T di = (T)i - c0, dj = (T)j - c0;
    T a = cs * di, b = sn * dj, c = sn * di, d = cs * dj;
    s1 = c0 + (a - b);
    s2 = c0 + (c + d);
  }
};

template <class T>
void imrotate_two(T* out, const T* img, T theta, int nx, bool adj, size_t stride) {
  if (!adj && std::fmod((double)theta, kTwoPi) == 0.0) {  // forward-only shortcut (rotatez.jl:341)
    for (int j = 0; j < nx; ++j)
      for (int i = 0; i < nx; ++i) out[i + j * stride] = img[i + j * stride];
    return;
  }
  Rot2<T> R(theta, nx);
  if (!adj) {
    for (int j = 0; j < nx; ++j)
      for (int i = 0; i < nx; ++i) {
        T s1, s2;
        R.pos(i, j, s1, s2);
        T f1 = std::floor(s1), f2 = std::floor(s2);
        int j1 = (int)f1, j2 = (int)f2;
        T t1 = s1 - f1, t2 = s2 - f2, u1 = T(1) - t1, u2 = T(1) - t2;
        auto at = [&](int a, int b) -> T {
          return (a >= 0 && a < nx && b >= 0 && b < nx) ? img[a + b * stride] : T(0);
        };
        T v = u1 * u2 * at(j1, j2);
        v += t1 * u2 * at(j1 + 1, j2);
        v += u1 * t2 * at(j1, j2 + 1);
        v += t1 * t2 * at(j1 + 1, j2 + 1);
        out[i + j * stride] = v;
      }
  } else {
    std::vector<T> acc((size_t)nx * nx, T(0));
    for (int j = 0; j < nx; ++j)
      for (int i = 0; i < nx; ++i) {
        T s1, s2;
        R.pos(i, j, s1, s2);
        T f1 = std::floor(s1), f2 = std::floor(s2);
        int j1 = (int)f1, j2 = (int)f2;
        T t1 = s1 - f1, t2 = s2 - f2, u1 = T(1) - t1, u2 = T(1) - t2;
        T x = img[i + j * stride];
        auto add = [&](int a, int b, T wgt) {
          if (a >= 0 && a < nx && b >= 0 && b < nx) acc[a + (size_t)b * nx] += wgt * x;
        };
        add(j1, j2, u1 * u2);
        add(j1 + 1, j2, t1 * u2);
        add(j1, j2 + 1, u1 * t2);
        add(j1 + 1, j2 + 1, t1 * t2);
      }
    for (int j = 0; j < nx; ++j)
      for (int i = 0; i < nx; ++i) out[i + j * stride] = acc[i + (size_t)j * nx];
  }
}

// ----------------------------------------------------------- plan --------
template <class T>
struct Plan {
  int nx, ny, nz, px, pz, nview, interp, nthread;
  T dy;
  const T* mumap;
  const T* psfs;  // [px,pz,ny,nview]
  std::vector<T> angle;
  // per-buffer (thread) work, mode :fast (src/spectplan.jl:95-112)
  std::vector<std::vector<T>> imgr, add_img, mumapr, expm;
  std::vector<RotWork<T>> rot;
  std::vector<PsfWork<T>> psf;
  Plan(int nx_, int nz_, int px_, int pz_, int nview_, const T* mu, const T* ps, T dy_, int interp_,
       const T* angles, int nthread_)
      : nx(nx_), ny(nx_), nz(nz_), px(px_), pz(pz_), nview(nview_), interp(interp_), nthread(nthread_),
        dy(dy_), mumap(mu), psfs(ps) {
    angle.resize(nview);
    for (int v = 0; v < nview; ++v) {
      if (angles) angle[v] = angles[v];
      else angle[v] = default_angle(v);
    }
    size_t N = (size_t)nx * ny * nz;
    for (int t = 0; t < nthread; ++t) {
      imgr.emplace_back(N);
      add_img.emplace_back(N);
      mumapr.emplace_back(N);
      expm.emplace_back((size_t)nx * nz);
      rot.emplace_back(nx);
      psf.emplace_back(nx, nz, px, pz);
    }
  }
  // viewangle = (0:nview-1)/nview * T(2pi), element rounded to T
  T default_angle(int v) const {
    double t2pi = (double)(T)kTwoPi;
    return (T)((double)v / nview * t2pi);
  }
  const T* psf_at(int y, int v) const { return psfs + ((size_t)v * ny + y) * px * pz; }
  void rotate(T* out, const T* in, T theta, int b, bool adj) {
    size_t s = nx;
    if (interp == 1) imrotate_one<T>(out, in, theta, rot[b], adj, s);
    else imrotate_two<T>(out, in, theta, nx, adj, s);
  }
  // exp_mumapr for plane y: exp(-dy * (-0.5 mu_y + sum_{j<=y} mu_j))
  // (src/project.jl:103-113, same summation order)
  void atten(int b, int y) {
    std::vector<T>& E = expm[b];
    const std::vector<T>& M = mumapr[b];
    for (int n = 0; n < nz; ++n)
      for (int m = 0; m < nx; ++m) E[m + (size_t)n * nx] = (T)(-0.5 * M[m + (size_t)nx * (y + (size_t)ny * n)]);
    for (int j = 0; j <= y; ++j)
      for (int n = 0; n < nz; ++n)
        for (int m = 0; m < nx; ++m) E[m + (size_t)n * nx] += M[m + (size_t)nx * (j + (size_t)ny * n)];
    for (auto& e : E) e = e * (-dy);
    for (auto& e : E) e = std::exp(e);
  }
  // project!(view, image, plan, buffer_id, viewidx) (src/project.jl:77-135)
  void project_view(T* view, const T* image, int b, int v) {
    size_t slice = (size_t)nx * ny;
    T* R = imgr[b].data();
    T* MU = mumapr[b].data();
    T* A = add_img[b].data();
    for (int z = 0; z < nz; ++z) {
      rotate(R + z * slice, image + z * slice, angle[v], b, false);
      rotate(MU + z * slice, mumap + z * slice, angle[v], b, false);
    }
    for (int y = 0; y < ny; ++y) {
      atten(b, y);
      const std::vector<T>& E = expm[b];
      for (int n = 0; n < nz; ++n)
        for (int m = 0; m < nx; ++m) R[m + nx * (y + (size_t)ny * n)] *= E[m + (size_t)n * nx];
      fft_conv<T>(A + (size_t)nx * y, R + (size_t)nx * y, psf_at(y, v), psf[b], slice, slice);
    }
    for (int n = 0; n < nz; ++n)
      for (int m = 0; m < nx; ++m) view[m + (size_t)n * nx] = A[m + nx * (0 + (size_t)ny * n)];
    for (int y = 1; y < ny; ++y)
      for (int n = 0; n < nz; ++n)
        for (int m = 0; m < nx; ++m) view[m + (size_t)n * nx] += A[m + nx * (y + (size_t)ny * n)];
  }
  // backproject!(image, view, plan, buffer_id, viewidx) (src/backproject.jl:69-124)
  void backproject_view(T* image, const T* view, int b, int v) {
    size_t slice = (size_t)nx * ny;
    T* R = imgr[b].data();
    T* MU = mumapr[b].data();
    for (int z = 0; z < nz; ++z) rotate(MU + z * slice, mumap + z * slice, angle[v], b, false);
    for (int y = 0; y < ny; ++y) {
      atten(b, y);
      fft_conv_adj<T>(R + (size_t)nx * y, view, psf_at(y, v), psf[b], slice, (size_t)nx);
      const std::vector<T>& E = expm[b];
      for (int n = 0; n < nz; ++n)
        for (int m = 0; m < nx; ++m) R[m + nx * (y + (size_t)ny * n)] *= E[m + (size_t)n * nx];
    }
    std::vector<T> tmp(slice);
    for (int z = 0; z < nz; ++z) {
      rotate(tmp.data(), R + z * slice, angle[v], b, true);
      std::memcpy(R + z * slice, tmp.data(), sizeof(T) * slice);
    }
    size_t N = slice * nz;
    for (size_t k = 0; k < N; ++k) image[k] += R[k];
  }
  // project!(views, image, plan; index) :fast (src/project.jl:143-163)
  void project(T* views, const T* image, const int* index, int nidx) {
    spawner(nthread, nidx, [&](int b, int ii) {
      project_view(views + (size_t)ii * nx * nz, image, b, index[ii]);
    });
  }
  // backproject!(image, views, plan; index) :fast (src/backproject.jl:132-162)
  void backproject(T* image, const T* views, const int* index, int nidx) {
    size_t N = (size_t)nx * ny * nz;
    std::fill(image, image + N, T(0));
    for (int t = 0; t < nthread; ++t) std::fill(add_img[t].begin(), add_img[t].end(), T(0));
    // add_img doubles as the per-buffer partial image; imgr is the work volume
    std::vector<std::vector<T>> part(nthread, std::vector<T>(N, T(0)));
    spawner(nthread, nidx, [&](int b, int ii) {
      backproject_view(part[b].data(), views + (size_t)ii * nx * nz, b, index[ii]);
    });
    for (int t = 0; t < nthread; ++t)
      for (size_t k = 0; k < N; ++k) image[k] += part[t][k];
  }
};

template <class T>
Plan<T>* make_plan(int nx, int nz, int px, int pz, int nview, const T* mumap, const T* psfs, T dy, int interp,
                   const T* angles, int nthread) {
  if (nthread < 1) nthread = 1;
  return new Plan<T>(nx, nz, px, pz, nview, mumap, psfs, dy, interp, angles, nthread);
}

// mlem! (src/ml-os-em.jl:21-49)
template <class T>
void mlem(T* out, const T* x0, const T* y, const T* bg, Plan<T>& P, int niter) {
  size_t N = (size_t)P.nx * P.ny * P.nz, M = (size_t)P.nx * P.nz * P.nview;
  std::vector<int> idx(P.nview);
  for (int v = 0; v < P.nview; ++v) idx[v] = v;
  std::vector<T> ones(M, T(1)), asum(N), ybar(M), yratio(M), back(N);
  P.backproject(asum.data(), ones.data(), idx.data(), P.nview);
  for (auto& a : asum)
    if (a == T(0)) a = (T)INFINITY;
  std::memcpy(out, x0, sizeof(T) * N);
  for (int it = 0; it < niter; ++it) {
    P.project(ybar.data(), out, idx.data(), P.nview);
    for (size_t k = 0; k < M; ++k) yratio[k] = y[k] / (ybar[k] + bg[k]);
    P.backproject(back.data(), yratio.data(), idx.data(), P.nview);
    for (size_t k = 0; k < N; ++k) out[k] *= back[k] / asum[k];
  }
}

// osem! with Ablock(plan, nblocks) subsets nb:nblocks:nview (src/ml-os-em.jl:70-131)
template <class T>
void osem(T* out, const T* x0, const T* y, const T* bg, Plan<T>& P, int nblocks, int niter) {
  size_t N = (size_t)P.nx * P.ny * P.nz, V = (size_t)P.nx * P.nz;
  int nsub = P.nview / nblocks;
  std::vector<std::vector<int>> idx(nblocks);
  for (int b = 0; b < nblocks; ++b)
    for (int v = b; v < P.nview; v += nblocks) idx[b].push_back(v);
  std::vector<std::vector<T>> asum(nblocks, std::vector<T>(N));
  std::vector<T> ones(V * nsub, T(1)), ybar(V * nsub), yratio(V * nsub), back(N);
  for (int b = 0; b < nblocks; ++b) {
    P.backproject(asum[b].data(), ones.data(), idx[b].data(), nsub);
    for (auto& a : asum[b])
      if (a == T(0)) a = (T)INFINITY;
  }
  std::memcpy(out, x0, sizeof(T) * N);
  for (int it = 0; it < niter; ++it)
    for (int b = 0; b < nblocks; ++b) {
      P.project(ybar.data(), out, idx[b].data(), nsub);
      for (int s = 0; s < nsub; ++s) {
        int v = idx[b][s];
        for (size_t k = 0; k < V; ++k)
          yratio[s * V + k] = y[(size_t)v * V + k] / (ybar[s * V + k] + bg[(size_t)v * V + k]);
      }
      P.backproject(back.data(), yratio.data(), idx[b].data(), nsub);
      for (size_t k = 0; k < N; ++k) out[k] *= back[k] / asum[b][k];
    }
}

}  // namespace

// ------------------------------------------------------- C exports ------
#define ORACLE_EXPORTS(T, SFX)                                                                              \
  extern "C" int oracle_project_##SFX(T* views, const T* image, const T* mumap, const T* psfs, int nx,    \
                                      int nz, int px, int pz, int nview, T dy, int interp, const T* angles, \
                                      const int* index, int nidx, int nthread) {                            \
    Plan<T>* P = make_plan<T>(nx, nz, px, pz, nview, mumap, psfs, dy, interp, angles, nthread);            \
    std::vector<int> all;                                                                                   \
    if (!index) {                                                                                           \
      for (int v = 0; v < nview; ++v) all.push_back(v);                                                     \
      index = all.data();                                                                                   \
      nidx = nview;                                                                                         \
    }                                                                                                       \
    P->project(views, image, index, nidx);                                                                  \
    delete P;                                                                                               \
    return 0;                                                                                               \
  }                                                                                                         \
  extern "C" int oracle_backproject_##SFX(T* image, const T* views, const T* mumap, const T* psfs, int nx, \
                                          int nz, int px, int pz, int nview, T dy, int interp,              \
                                          const T* angles, const int* index, int nidx, int nthread) {       \
    Plan<T>* P = make_plan<T>(nx, nz, px, pz, nview, mumap, psfs, dy, interp, angles, nthread);            \
    std::vector<int> all;                                                                                   \
    if (!index) {                                                                                           \
      for (int v = 0; v < nview; ++v) all.push_back(v);                                                     \
      index = all.data();                                                                                   \
      nidx = nview;                                                                                         \
    }                                                                                                       \
    P->backproject(image, views, index, nidx);                                                              \
    delete P;                                                                                               \
    return 0;                                                                                               \
  }                                                                                                         \
  extern "C" int oracle_mlem_##SFX(T* out, const T* x0, const T* y, const T* bg, const T* mumap,           \
                                   const T* psfs, int nx, int nz, int px, int pz, int nview, T dy,          \
                                   int interp, const T* angles, int niter, int nthread) {                   \
    Plan<T>* P = make_plan<T>(nx, nz, px, pz, nview, mumap, psfs, dy, interp, angles, nthread);            \
    mlem<T>(out, x0, y, bg, *P, niter);                                                                     \
    delete P;                                                                                               \
    return 0;                                                                                               \
  }                                                                                                         \
  extern "C" int oracle_osem_##SFX(T* out, const T* x0, const T* y, const T* bg, const T* mumap,           \
                                   const T* psfs, int nx, int nz, int px, int pz, int nview, T dy,          \
                                   int interp, const T* angles, int nblocks, int niter, int nthread) {      \
    if (nblocks < 1 || nview % nblocks != 0) return -1;                                                     \
    Plan<T>* P = make_plan<T>(nx, nz, px, pz, nview, mumap, psfs, dy, interp, angles, nthread);            \
    osem<T>(out, x0, y, bg, *P, nblocks, niter);                                                            \
    delete P;                                                                                               \
    return 0;                                                                                               \
  }                                                                                                         \
  extern "C" int oracle_imrotate_##SFX(T* out, const T* img, int nx, T theta, int interp, int adj) {       \
    if (interp == 1) {                                                                                      \
      RotWork<T> w(nx);                                                                                     \
      imrotate_one<T>(out, img, theta, w, adj != 0, (size_t)nx);                                            \
    } else {                                                                                                \
      imrotate_two<T>(out, img, theta, nx, adj != 0, (size_t)nx);                                           \
    }                                                                                                       \
    return 0;                                                                                               \
  }                                                                                                         \
  extern "C" int oracle_fft_conv_##SFX(T* out, const T* img, int nx, int nz, const T* ker, int px, int pz, \
                                       int adj) {                                                           \
    PsfWork<T> w(nx, nz, px, pz);                                                                           \
    if (adj) fft_conv_adj<T>(out, img, ker, w, (size_t)nx, (size_t)nx);                                     \
    else fft_conv<T>(out, img, ker, w, (size_t)nx, (size_t)nx);                                             \
    return 0;                                                                                               \
  }                                                                                                         \
  extern "C" int oracle_rot_f90_##SFX(T* out, const T* img, int L, int m, int adj) {                       \
    return rot_f90<T>(out, img, L, m, adj != 0);                                                            \
  }                                                                                                         \
  extern "C" T oracle_default_angle_##SFX(int v, int nview) {                                               \
    double t2pi = (double)(T)kTwoPi;                                                                        \
    return (T)((double)v / nview * t2pi);                                                                   \
  }

ORACLE_EXPORTS(float, f32)
ORACLE_EXPORTS(double, f64)

// Padding / shift helpers, exported for the known-answer tests of
// test/helper.jl (float only, like those tests).
extern "C" void oracle_padzero_f32(float* out, const float* img, int M, int N, int up, int down, int left,
                                   int right) {  // src/helper.jl:20-34
  int P = M + up + down, Q = N + left + right;
  std::fill(out, out + (size_t)P * Q, 0.0f);
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < M; ++i) out[(up + i) + (size_t)(left + j) * P] = img[i + (size_t)j * M];
}
extern "C" void oracle_padrepl_f32(float* out, const float* img, int M, int N, int up, int down, int left,
                                   int right) {  // src/helper.jl:42-55
  int P = M + up + down, Q = N + left + right;
  for (int j = 0; j < Q; ++j)
    for (int i = 0; i < P; ++i)
      out[i + (size_t)j * P] = img[clampi(i - up, 0, M - 1) + (size_t)clampi(j - left, 0, N - 1) * M];
}
extern "C" void oracle_pad2sizezero_f32(float* out, const float* img, int M, int N, int P,
                                        int Q) {  // src/helper.jl:66-80
  int pd1 = (P - M + 1) / 2, pd2 = (Q - N + 1) / 2;
  std::fill(out, out + (size_t)P * Q, 0.0f);
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < M; ++i) out[(pd1 + i) + (size_t)(pd2 + j) * P] = img[i + (size_t)j * M];
}
extern "C" int oracle_fftshift2_f32(float* dst, const float* src, int M, int N) {  // src/helper.jl:111-142
  if (N == 1) {
    if (M % 2) return -1;
    int m = M / 2;
    for (int i = 0; i < m; ++i) {
      dst[i] = src[m + i];
      dst[i + m] = src[i];
    }
    return 0;
  }
  if ((M % 2) || (N % 2)) return -1;
  int m = M / 2, n = N / 2;
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < M; ++i) dst[i + (size_t)j * M] = src[(i + m) % M + (size_t)((j + n) % N) * M];
  return 0;
}
extern "C" int oracle_rot_padsize(int nx) { return rot_padsize(nx); }
extern "C" int oracle_power2(int x) { return power2(x); }
