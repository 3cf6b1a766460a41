// The :gradepro estimator on the device: bandwidth ladder, per-step propagation +
// inverse FFT + variance-to-mean ratio + bootstrap variance, means, and the per-point
// convergence state machine.
//
// Reference (ParallelKDE.jl): src/DensityEstimators/GradeProEstimator.jl:700-1089,
// src/StatisticsPropagation/DirectSpace.jl:526-1111, FourierSpace.jl:122-524.
//
// Layout on the device:
//   spectra  : [z_0, w_0, z_1, w_1, ..., z_{P-1}, w_{P-1}, z_F], G complex FP64 each, with
//              z_p = FFT(M_{2p} + i M_{2p+1}), w_p = FFT(V_{2p} + i V_{2p+1}) (bootstrap
//              pairs share one complex transform; the two halves have equal magnitude,
//              so neither loses precision to the other) and z_F = FFT(M_full).
//   scratch  : per-step inverse-FFT intermediates of a group of pairs.
//   welford  : per-point (mean, m2) over bootstraps, FP64.
//   state    : f_prev1, f_prev2, minima (FP64), counters_low/over (u16), flags (u8),
//              density (FP64), selected step (i32), final-step means (FP64).
#include <algorithm>
#include <cstring>
#include <limits>

#include "pkde_internal.cuh"
#include "pkde_step.cuh"

namespace pkde {

void dirac_paired(pkde_ctx *ctx, const pkde_grid *g, const double *d_data, int64_t n, const int32_t *d_idx,
                  int64_t nboot, uint64_t seed, double2 *spectra, cudaStream_t st);
int lines_per_cta(int n, int64_t nlines);

namespace {

constexpr int kThreads = 256;

// ------------------------------------------------------------------- convergence
__global__ void converge_kernel(int64_t G, double *density, const double *means, const double *f, const double *f1,
                                const double *f2, double dlogt, double eps, int64_t steps_low, int64_t steps_over,
                                double *minima, uint16_t *c_low, uint16_t *c_over, uint8_t *flags) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < G; i += (int64_t)gridDim.x * blockDim.x) {
    StabilityResult r = find_stability(f[i], f1[i], f2[i], dlogt, eps, steps_low, steps_over, minima[i], c_low[i],
                                  c_over[i], flags[i]);
    c_low[i] = r.c_low;
    c_over[i] = r.c_over;
    flags[i] = r.flag;
    minima[i] = r.new_min;
    if (r.more_stable) density[i] = means[i];
  }
}

// calculate_scaled_vmr! on complex inputs (DirectSpace.jl:526-584): |.| = sqrt(re^2+im^2).
__global__ void scaled_vmr_kernel(int64_t G, int nboot, const double2 *sk, const double2 *s2k, double n_samples,
                                  double scaling, double *out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < G; i += (int64_t)gridDim.x * blockDim.x) {
    double mean = 0.0, m2 = 0.0;
    for (int b = 0; b < nboot; ++b) {
      double2 a = sk[b * G + i], c = s2k[b * G + i];
      double m = __ddiv_rn(sqrt(__dadd_rn(__dmul_rn(a.x, a.x), __dmul_rn(a.y, a.y))), n_samples);
      double v = __dsub_rn(__ddiv_rn(sqrt(__dadd_rn(__dmul_rn(c.x, c.x), __dmul_rn(c.y, c.y))), n_samples),
                           __dmul_rn(m, m));
      double x = __ddiv_rn(v, m);
      double delta = __dsub_rn(x, mean);
      mean = __dadd_rn(mean, __ddiv_rn(delta, (double)(b + 1)));
      m2 = __dadd_rn(m2, __dmul_rn(delta, __dsub_rn(x, mean)));
    }
    double v = __ddiv_rn(__dmul_rn(scaling, m2), (double)(nboot - 1));
    out[i] = isfinite(v) ? log(v) : nan("");
  }
}

// ------------------------------------------------------------- fused final pass
// Inverse FFT along grid axis 1 of the z/w rows of one group of bootstrap pairs, then
// per point: m = |M|/n, v = |V|/n - m^2, r = v/m for both bootstraps of each pair and
// the Welford update over bootstraps in order (DirectSpace.jl:544-581).
template <int PPT>
__global__ void __launch_bounds__(kThreads) vmr_axis1_kernel(
    const double2 *__restrict__ in, int npairs, int b0, int nboot, int n1, int64_t rows, FftPlan plan,
    const double2 *__restrict__ tw, const double *__restrict__ fz, const double *__restrict__ fw, double cz, double cw,
    double n_samples, int64_t G, double *__restrict__ wmean, double *__restrict__ wm2, int first, int tl, int pitch) {
  extern __shared__ double2 smem[];
  double2 *bufA = smem;
  double2 *bufB = smem + (size_t)tl * pitch;
  const int64_t r0 = (int64_t)blockIdx.x * tl;
  const int nl = (int)min((int64_t)tl, rows - r0);
  const int npts = nl * n1;
  double mean[PPT], m2[PPT];
#pragma unroll
  for (int q = 0; q < PPT; ++q) {
    const int e = threadIdx.x + q * kThreads;
    const int64_t gi = r0 * n1 + e;
    if (!first && e < npts) {
      mean[q] = wmean[gi];
      m2[q] = wm2[gi];
    } else {
      mean[q] = 0.0;
      m2[q] = 0.0;
    }
  }
  for (int p = 0; p < npairs; ++p) {
    double2 zval[PPT];
    for (int arr = 0; arr < 2; ++arr) {
      const double2 *src = in + (int64_t)(2 * p + arr) * G + r0 * n1;
      const double *f = arr ? fw : fz;
      const double c = arr ? cw : cz;
      for (int e = threadIdx.x; e < npts; e += kThreads) {
        const int k = e % n1;
        bufA[(e / n1) * pitch + k] = cscale(src[e], c * f[k]);
      }
      __syncthreads();
      double2 *res = smem_fft<1>(bufA, bufB, pitch, nl, plan, tw);
      if (arr == 0) {
#pragma unroll
        for (int q = 0; q < PPT; ++q) {
          const int e = threadIdx.x + q * kThreads;
          if (e < npts) zval[q] = res[(e / n1) * pitch + (e % n1)];
        }
      } else {
        const int bA = b0 + 2 * p;
#pragma unroll
        for (int q = 0; q < PPT; ++q) {
          const int e = threadIdx.x + q * kThreads;
          if (e < npts) {
            const double2 w = res[(e / n1) * pitch + (e % n1)];
            // bootstrap bA from the real parts, bA + 1 from the imaginary parts
            for (int h = 0; h < 2; ++h) {
              const int b = bA + h;
              if (b >= nboot) break;
              const double Mv = h ? zval[q].y : zval[q].x;
              const double Vv = h ? w.y : w.x;
              const double m = __ddiv_rn(fabs(Mv), n_samples);
              const double v = __dsub_rn(__ddiv_rn(fabs(Vv), n_samples), __dmul_rn(m, m));
              const double x = __ddiv_rn(v, m);
              const double delta = __dsub_rn(x, mean[q]);
              mean[q] = __dadd_rn(mean[q], __ddiv_rn(delta, (double)(b + 1)));
              m2[q] = __dadd_rn(m2[q], __dmul_rn(delta, __dsub_rn(x, mean[q])));
            }
          }
        }
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int q = 0; q < PPT; ++q) {
    const int e = threadIdx.x + q * kThreads;
    if (e < npts) {
      wmean[r0 * n1 + e] = mean[q];
      wm2[r0 * n1 + e] = m2[q];
    }
  }
}

using ConvState = StepState;

// Means of the full sample (DirectSpace.jl:747-764) for one step, the scaled VMR
// variance from the Welford state (:579-580), and the convergence update
// (GradeProEstimator.jl:638-669).  Generic line lengths.
template <int PPT>
__global__ void __launch_bounds__(kThreads) means_converge_kernel(
    const double2 *__restrict__ in, int n1, int64_t rows, FftPlan plan, const double2 *__restrict__ tw,
    const double *__restrict__ fz, double cz, const double *__restrict__ wm2, double vscale, double bm1, double dlogt,
    double eps, int64_t steps_low, int64_t steps_over, ConvState cs, int step, int tl, int pitch) {
  extern __shared__ double2 smem[];
  double2 *bufA = smem;
  double2 *bufB = smem + (size_t)tl * pitch;
  const int64_t r0 = (int64_t)blockIdx.x * tl;
  const int nl = (int)min((int64_t)tl, rows - r0);
  const int npts = nl * n1;
  const double2 *src = in + r0 * n1;
  for (int e = threadIdx.x; e < npts; e += kThreads) {
    const int k = e % n1;
    bufA[(e / n1) * pitch + k] = cscale(src[e], cz * fz[k]);
  }
  __syncthreads();
  double2 *res = smem_fft<1>(bufA, bufB, pitch, nl, plan, tw);
  for (int e = threadIdx.x; e < npts; e += kThreads) {
    const int64_t i = r0 * n1 + e;
    const double2 z = res[(e / n1) * pitch + (e % n1)];
    const double mu = sqrt(__dadd_rn(__dmul_rn(z.x, z.x), __dmul_rn(z.y, z.y)));
    step_update(cs, i, mu, __ddiv_rn(__dmul_rn(vscale, wm2[i]), bm1), dlogt, eps, steps_low, steps_over, step);
  }
}

__global__ void init_state_kernel(int64_t G, ConvState cs) {
  const double qnan = nan("");
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < G; i += (int64_t)gridDim.x * blockDim.x) {
    cs.f1[i] = qnan;
    cs.f2[i] = qnan;
    cs.minima[i] = qnan;
    cs.density[i] = qnan;
    cs.c_low[i] = 0;
    cs.c_over[i] = 0;
    cs.flags[i] = 0;
    cs.selected[i] = -1;
  }
}

// replace_nans! (GradeProEstimator.jl:1053-1072).
__global__ void replace_nans_kernel(int64_t G, ConvState cs, int nsteps_total) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < G; i += (int64_t)gridDim.x * blockDim.x) {
    if (isnan(cs.density[i])) cs.density[i] = cs.mu_last[i];
    if (cs.selected[i] < 0) cs.selected[i] = nsteps_total;
  }
}

// Deterministic per-axis sums of x (mean == nullptr) or of (x - mean)^2: each block
// writes its partial sums (fixed tree order), a single block adds the partials in order.
__device__ __forceinline__ double block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
  return t;
}

__global__ void moments_partial_kernel(const double *data, int64_t n, int ndim, const double *mean, double *partial) {
  __shared__ double sh[32];
  for (int j = 0; j < ndim; ++j) {
    const double mu = mean ? mean[j] : 0.0;
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
      const double x = data[i * ndim + j];
      s += mean ? (x - mu) * (x - mu) : x;
    }
    const double t = block_sum(s, sh);
    if (threadIdx.x == 0) partial[blockIdx.x * ndim + j] = t;
  }
}

__global__ void moments_final_kernel(const double *partial, int nblocks, int ndim, double *out) {
  if (threadIdx.x < ndim) {
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += partial[b * ndim + threadIdx.x];
    out[threadIdx.x] = s;
  }
}

int blocks_for(pkde_ctx *ctx, int64_t work) {
  int64_t b = (work + kThreads - 1) / kThreads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)ctx->sm_count * 8));
}

}  // namespace

// ---------------------------------------------------------------- bandwidth ladder
// get_time (GradeProEstimator.jl:860-905), calculate_duration_steps (:954-966),
// calculate_dlogt (:1074-1089), defaults (:705, 754-766, 541-550).
struct Ladder {
  int ndim;
  int64_t S;                  // number of bandwidths (n_steps + 1)
  std::vector<double> times;  // S x ndim
  double t0[4];
  int64_t steps_low, steps_over;
  double eps;
  std::vector<double> dlogt;  // S
  std::vector<double> vscale; // S: prod(t^2+t0^2)^(3/2) n^3
  std::vector<double> cw;     // S: prod(t0) / sqrt(prod(t0^2 + t^2))
};

static double fold_prod(const double *v, int n) {
  double p = v[0];
  for (int j = 1; j < n; ++j) p = p * v[j];
  return p;
}

Ladder make_ladder(const pkde_gradepro_params *p, const double *bw_final, int64_t n_samples) {
  Ladder L{};
  const int N = p->grid.ndim;
  L.ndim = N;
  const double nan = std::numeric_limits<double>::quiet_NaN();
  double alpha_s = std::isnan(p->alpha_s) ? (N == 1 ? 0.0 : 0.06) : p->alpha_s;
  double alpha_os = std::isnan(p->alpha_os) ? 0.1 : p->alpha_os;
  L.eps = std::isnan(p->eps) ? (N == 1 ? 2.0 : -0.5) : p->eps;
  double dt[4];
  double nsteps_d;
  if (p->n_steps > 0 || std::isnan(p->bw_step)) {
    const int64_t ns = p->n_steps > 0 ? p->n_steps : 250;
    for (int j = 0; j < N; ++j) dt[j] = bw_final[j] / (double)ns;
    nsteps_d = (double)ns;
  } else {
    double m = std::numeric_limits<double>::infinity();
    for (int j = 0; j < N; ++j) {
      dt[j] = p->bw_step;
      if (p->bw_step > bw_final[j] || p->bw_step <= 0) throw invalid("Invalid time step");
      m = std::min(m, std::floor(bw_final[j] / p->bw_step));
    }
    nsteps_d = m;
  }
  if (!(nsteps_d >= 1) || nsteps_d > 65535) throw invalid("number of bandwidth steps must be in 1..65535");
  L.S = (int64_t)nsteps_d + 1;
  L.times.resize(L.S * N);
  for (int64_t s = 0; s < L.S; ++s)
    for (int j = 0; j < N; ++j) L.times[s * N + j] = dt[j] * (double)s;
  if (alpha_s < 0 || alpha_s > 1 || alpha_os < 0 || alpha_os > 1) throw invalid("Fraction must be in the range [0, 1]");
  double sb = 0.0, so = 0.0;
  for (int j = 0; j < N; ++j) {
    const double ns = L.times[(L.S - 1) * N + j] / dt[j];
    sb = (j == 0) ? alpha_s * ns : sb + alpha_s * ns;
    so = (j == 0) ? alpha_os * ns : so + alpha_os * ns;
  }
  L.steps_low = (int64_t)std::nearbyint(sb / N);
  L.steps_over = (int64_t)std::nearbyint(so / N);
  double t0sq[4], tmp[4];
  for (int j = 0; j < N; ++j) {
    L.t0[j] = p->grid.h[j] / 2;
    t0sq[j] = L.t0[j] * L.t0[j];
  }
  const long double n3 = (long double)n_samples * (long double)n_samples * (long double)n_samples;
  const double n3d = (double)n3;  // n^3 rounded once (exact in long double up to 2^64)
  const int64_t B = p->n_bootstraps;
  L.dlogt.resize(L.S);
  L.vscale.resize(L.S);
  L.cw.resize(L.S);
  const double det_t0 = fold_prod(L.t0, N);
  for (int64_t s = 0; s < L.S; ++s) {
    const double *t = &L.times[s * N];
    for (int j = 0; j < N; ++j) tmp[j] = t0sq[j] + t[j] * t[j];
    const double det_curr = fold_prod(tmp, N);
    double det_prev;
    if (s == 0) {
      det_prev = fold_prod(t0sq, N);
    } else {
      const double *tp = &L.times[(s - 1) * N];
      for (int j = 0; j < N; ++j) tmp[j] = t0sq[j] + tp[j] * tp[j];
      det_prev = fold_prod(tmp, N);
    }
    L.dlogt[s] = std::log(det_curr / det_prev);
    for (int j = 0; j < N; ++j) tmp[j] = t[j] * t[j] + t0sq[j];
    const double scaling = std::pow(fold_prod(tmp, N), 1.5) * n3d;
    L.vscale[s] = scaling;
    L.cw[s] = det_t0 / std::sqrt(det_curr);
  }
  (void)nan;
  return L;
}

// Silverman's rule (DirectSpace.jl:1102-1111) from FP64 device moments.
static void silverman_device(pkde_ctx *ctx, const double *d_data, int64_t n, int N, double *bw, cudaStream_t st) {
  const int nb = blocks_for(ctx, n);
  double *m = (double *)ensure(ctx, BUF_MISC, sizeof(double) * (16 + 4 * (size_t)nb));
  double *sum = m, *cen = m + 4, *meanv = m + 8, *partial = m + 16;
  {
    ::pkde::Trace _tr(ctx, PKDE_PHASE_OTHER, st);
    moments_partial_kernel<<<nb, kThreads, 0, st>>>(d_data, n, N, nullptr, partial);
  }
  PKDE_CHECK_LAUNCH();
  {
    ::pkde::Trace _tr(ctx, PKDE_PHASE_OTHER, st);
    moments_final_kernel<<<1, 32, 0, st>>>(partial, nb, N, sum);
  }
  PKDE_CHECK_LAUNCH();
  double h[4];
  PKDE_CUDA_TRY(cudaMemcpyAsync(h, sum, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  PKDE_CUDA_TRY(cudaStreamSynchronize(st));
  for (int j = 0; j < N; ++j) h[j] /= (double)n;
  PKDE_CUDA_TRY(cudaMemcpyAsync(meanv, h, sizeof(double) * N, cudaMemcpyHostToDevice, st));
  {
    ::pkde::Trace _tr(ctx, PKDE_PHASE_OTHER, st);
    moments_partial_kernel<<<nb, kThreads, 0, st>>>(d_data, n, N, meanv, partial);
  }
  PKDE_CHECK_LAUNCH();
  {
    ::pkde::Trace _tr(ctx, PKDE_PHASE_OTHER, st);
    moments_final_kernel<<<1, 32, 0, st>>>(partial, nb, N, cen);
  }
  PKDE_CHECK_LAUNCH();
  double c[4];
  PKDE_CUDA_TRY(cudaMemcpyAsync(c, cen, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  PKDE_CUDA_TRY(cudaStreamSynchronize(st));
  const double pref = std::pow(4.0 / ((double)(N + 2) * (double)n), 1.0 / (double)(N + 4));
  for (int j = 0; j < N; ++j) bw[j] = pref * std::sqrt(c[j] / (double)(n - 1));
}

// Per-step, per-axis propagation factors: p(k) = exp(-0.5 (k t)^2) and sqrt(p(k)),
// k = m * (2 pi ((1/h)/n)) with fftfreq ordering (Grids.jl:225-231).
static void factor_tables(const pkde_grid *g, const Ladder &L, std::vector<double> &fz, std::vector<double> &fw,
                          std::vector<int64_t> &axis_off) {
  const int N = g->ndim;
  int64_t tot = 0;
  axis_off.assign(N + 1, 0);
  for (int j = 0; j < N; ++j) {
    axis_off[j] = tot;
    tot += g->dims[j];
  }
  axis_off[N] = tot;
  fz.assign(L.S * tot, 0.0);
  fw.assign(L.S * tot, 0.0);
  const double two_pi = 6.283185307179586;
  for (int64_t s = 0; s < L.S; ++s) {
    for (int j = 0; j < N; ++j) {
      const int64_t n = g->dims[j];
      const double mult = two_pi * ((1.0 / g->h[j]) / (double)n);
      const double t = L.times[s * N + j];
      const int64_t nneg = (n - 1) / 2 + 1;
      for (int64_t m = 0; m < n; ++m) {
        const double mm = (double)(m < nneg ? m : m - n);
        const double kt = (mm * mult) * t;
        const double pv = std::exp(-0.5 * (kt * kt));
        fz[s * tot + axis_off[j] + m] = pv;
        fw[s * tot + axis_off[j] + m] = std::sqrt(pv);
      }
    }
  }
}

template <class K>
static void set_smem(K kernel, size_t bytes) {
  PKDE_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

// The plain one-estimation-at-a-time pipeline.
struct Estimation {
  const pkde_gradepro_params *p;
  int64_t n;
  const double *d_data;
  const int32_t *d_idx;
  uint64_t seed;
};

void run_gradepro(pkde_ctx *ctx, const Estimation &E, double *d_density, int32_t *d_selected, cudaStream_t st) {
  const pkde_gradepro_params *p = E.p;
  const pkde_grid *g = &p->grid;
  const int N = g->ndim;
  const int64_t G = grid_size(g);
  const int64_t B = p->n_bootstraps;
  const int64_t npairs = (B + 1) / 2;
  const int n1 = (int)g->dims[0];
  const int64_t rows = G / n1;

  // bandwidth ladder (host), Silverman from device moments when bw_final is NaN
  double bw[4];
  bool need_silverman = false;
  for (int j = 0; j < N; ++j) need_silverman |= std::isnan(p->bw_final[j]);
  if (need_silverman) silverman_device(ctx, E.d_data, E.n, N, bw, st);
  for (int j = 0; j < N; ++j)
    if (!std::isnan(p->bw_final[j])) bw[j] = p->bw_final[j];
  Ladder L = make_ladder(p, bw, E.n);

  // device buffers
  double2 *spectra = (double2 *)ensure(ctx, BUF_SPECTRA, sizeof(double2) * (2 * npairs + 1) * G);
  const int64_t pair_bytes = (int64_t)sizeof(double2) * 2 * G;
  int64_t group = std::max<int64_t>(1, std::min<int64_t>(npairs, (48ll << 20) / pair_bytes));
  if (N == 1) group = npairs;
  double2 *scratch = (double2 *)ensure(ctx, BUF_SCRATCH, N > 1 ? (size_t)pair_bytes * group : 16);
  double *wel = (double *)ensure(ctx, BUF_WELFORD, sizeof(double) * 2 * G);
  double *wmean = wel, *wm2 = wel + G;
  char *stb = (char *)ensure(ctx, BUF_STATE, (sizeof(double) * 5 + sizeof(uint16_t) * 2 + 1 + 4) * G + 256);
  ConvState cs;
  cs.f1 = (double *)stb;
  cs.f2 = cs.f1 + G;
  cs.minima = cs.f2 + G;
  cs.density = cs.minima + G;
  cs.mu_last = cs.density + G;
  cs.selected = (int32_t *)(cs.mu_last + G);
  cs.c_low = (uint16_t *)(cs.selected + G);
  cs.c_over = cs.c_low + G;
  cs.flags = (uint8_t *)(cs.c_over + G);

  std::vector<double> fz, fw;
  std::vector<int64_t> aoff;
  factor_tables(g, L, fz, fw, aoff);
  const int64_t tot = aoff[N];
  double *tables = (double *)ensure(ctx, BUF_TABLES, sizeof(double) * 2 * L.S * tot);
  PKDE_CUDA_TRY(cudaMemcpyAsync(tables, fz.data(), sizeof(double) * L.S * tot, cudaMemcpyHostToDevice, st));
  PKDE_CUDA_TRY(cudaMemcpyAsync(tables + L.S * tot, fw.data(), sizeof(double) * L.S * tot, cudaMemcpyHostToDevice, st));
  const double *dfz = tables, *dfw = tables + L.S * tot;

  // binning into the paired layout, forward FFT of every array
  dirac_paired(ctx, g, E.d_data, E.n, E.d_idx, B, E.seed, spectra, st);
  fft_nd(ctx, N, g->dims, spectra, 2 * npairs + 1, -1, st, PKDE_PHASE_FORWARD_FFT);

  if (steps1d_ok(g)) {
    // 1-D: every bandwidth step in parallel (one CTA each), then the convergence
    // state machine over the stored per-step f_s and means.
    const int64_t S = L.S;
    double *per_step = (double *)ensure(ctx, BUF_SCRATCH, sizeof(double) * (2 * S * G + 3 * S));
    double *f_all = per_step, *mu_all = per_step + S * G;
    double *d_cw = mu_all + S * G, *d_vs = d_cw + S, *d_dl = d_vs + S;
    PKDE_CUDA_TRY(cudaMemcpyAsync(d_cw, L.cw.data(), sizeof(double) * S, cudaMemcpyHostToDevice, st));
    PKDE_CUDA_TRY(cudaMemcpyAsync(d_vs, L.vscale.data(), sizeof(double) * S, cudaMemcpyHostToDevice, st));
    PKDE_CUDA_TRY(cudaMemcpyAsync(d_dl, L.dlogt.data(), sizeof(double) * S, cudaMemcpyHostToDevice, st));
    steps1d(ctx, n1, spectra, (int)npairs, (int)B, (int)S, dfz, dfw, tot, d_cw, 1.0 / (double)G, 1.0 / (double)E.n,
            d_vs, f_all, mu_all, st);
    converge_steps(ctx, G, (int)S, f_all, mu_all, d_dl, L.eps, L.steps_low, L.steps_over, cs, st);
    if (d_density) PKDE_CUDA_TRY(cudaMemcpyAsync(d_density, cs.density, sizeof(double) * G, cudaMemcpyDeviceToDevice, st));
    if (d_selected)
      PKDE_CUDA_TRY(cudaMemcpyAsync(d_selected, cs.selected, sizeof(int32_t) * G, cudaMemcpyDeviceToDevice, st));
    return;
  }

  {
    ::pkde::Trace _tr(ctx, PKDE_PHASE_OTHER, st);
    init_state_kernel<<<blocks_for(ctx, G), kThreads, 0, st>>>(G, cs);
  }
  PKDE_CHECK_LAUNCH();

  if (engine_ok(g)) {
    // N-D on power-of-two axes: the persistent step engine runs every bandwidth step
    EngineArgs A{};
    A.grid = g;
    A.npairs = (int)npairs;
    A.nboot = (int)B;
    A.S = (int)L.S;
    A.spectra = spectra;
    A.fz = dfz;
    A.fw = dfw;
    A.tab_stride = tot;
    for (int j = 0; j < N; ++j) A.aoff[j] = aoff[j];
    A.cw = L.cw.data();
    A.vscale = L.vscale.data();
    A.dlogt = L.dlogt.data();
    A.inv_n = 1.0 / (double)E.n;
    A.eps = L.eps;
    A.steps_low = L.steps_low;
    A.steps_over = L.steps_over;
    A.cs = cs;
    run_engine(ctx, A, st);
    {
      ::pkde::Trace _tr(ctx, PKDE_PHASE_OTHER, st);
      replace_nans_kernel<<<blocks_for(ctx, G), kThreads, 0, st>>>(G, cs, (int)L.S);
    }
    PKDE_CHECK_LAUNCH();
    if (d_density) PKDE_CUDA_TRY(cudaMemcpyAsync(d_density, cs.density, sizeof(double) * G, cudaMemcpyDeviceToDevice, st));
    if (d_selected)
      PKDE_CUDA_TRY(cudaMemcpyAsync(d_selected, cs.selected, sizeof(int32_t) * G, cudaMemcpyDeviceToDevice, st));
    return;
  }

  // final-pass geometry
  int tl = std::max(1, std::min<int>(2048 / n1, 16));
  if (tl > rows) tl = (int)rows;
  const int ppt_needed = (tl * n1 + kThreads - 1) / kThreads;
  const int pitch = n1 + 1;
  const size_t smem = sizeof(double2) * 2 * (size_t)tl * pitch;
  if (smem > ctx->smem_optin) throw Error{PKDE_EUNSUPPORTED, "grid axis 1 too long for the shared-memory FFT"};
  FftPlan plan1 = make_plan(n1);
  const double2 *tw1 = twiddles_device(ctx, n1);
  const unsigned fblocks = (unsigned)((rows + tl - 1) / tl);
  const double invG = 1.0 / (double)G;
  const double nsd = (double)E.n;

  auto launch_vmr = [&](const double2 *in, int np, int b0, int first, const double *fz1, const double *fw1, double cz,
                        double cw) {
#define PKDE_VMR_CASE(P)                                                                                   \
  if (ppt_needed <= P) {                                                                                   \
    set_smem(vmr_axis1_kernel<P>, smem);                                                                   \
    { \
      ::pkde::Trace _tr(ctx, PKDE_PHASE_STEP_VMR, st); \
      vmr_axis1_kernel<P><<<fblocks, kThreads, smem, st>>>(in, np, b0, (int)B, n1, rows, plan1, tw1, fz1,   \
                                                           fw1, cz, cw, nsd, G, wmean, wm2, first, tl, pitch); \
    } \
    PKDE_CHECK_LAUNCH();                                                                                   \
    return;                                                                                                \
  }
    PKDE_VMR_CASE(8)
    PKDE_VMR_CASE(16)
    PKDE_VMR_CASE(24)
#undef PKDE_VMR_CASE
    throw Error{PKDE_EUNSUPPORTED, "grid axis 1 too long"};
  };
  auto launch_means = [&](const double2 *in, const double *fz1, double cz, int64_t s) {
#define PKDE_MEANS_CASE(P)                                                                                    \
  if (ppt_needed <= P) {                                                                                      \
    set_smem(means_converge_kernel<P>, smem);                                                                 \
    { \
      ::pkde::Trace _tr(ctx, PKDE_PHASE_STEP_MEANS, st); \
      means_converge_kernel<P><<<fblocks, kThreads, smem, st>>>(in, n1, rows, plan1, tw1, fz1, cz, wm2,        \
                                                                L.vscale[s], (double)(B - 1), L.dlogt[s], L.eps, L.steps_low,    \
                                                                L.steps_over, cs, (int)s, tl, pitch);           \
    } \
    PKDE_CHECK_LAUNCH();                                                                                      \
    return;                                                                                                   \
  }
    PKDE_MEANS_CASE(8)
    PKDE_MEANS_CASE(16)
    PKDE_MEANS_CASE(24)
#undef PKDE_MEANS_CASE
    throw Error{PKDE_EUNSUPPORTED, "grid axis 1 too long"};
  };

  const bool pow2 = N > 1 && pow2_path_ok(g);
  const double inv_n = 1.0 / nsd;
  for (int64_t s = 0; s < L.S; ++s) {
    const double *fzs = dfz + s * tot, *fws = dfw + s * tot;
    for (int64_t p0 = 0; p0 < npairs; p0 += group) {
      const int np = (int)std::min<int64_t>(group, npairs - p0);
      const double2 *src = spectra + 2 * p0 * G;
      if (N > 1) {
        // axes N..2 on the group's z/w arrays, propagation factor applied on the first load
        for (int a = N - 1; a >= 1; --a) {
          LineSet ls = axis_lines(N, g->dims, a, 2 * np);
          const double *facs[2] = {fzs + aoff[a], fws + aoff[a]};
          const double ones[2] = {1.0, 1.0};
          if (pow2)
            axis_pass_pow2(ctx, ls, a == N - 1 ? src : scratch, scratch, facs, ones, 2, st);
          else
            fft_axis(ctx, ls, a == N - 1 ? src : scratch, scratch, 1, facs, ones, 2, st, PKDE_PHASE_STEP_FFT);
        }
        src = scratch;
      }
      if (pow2)
        vmr_pass_pow2(ctx, n1, src, np, (int)(2 * p0), (int)B, rows, fzs + aoff[0], fws + aoff[0], invG,
                      invG * L.cw[s], inv_n, G, wel, p0 == 0 ? 1 : 0, st);
      else
        launch_vmr(src, np, (int)(2 * p0), p0 == 0 ? 1 : 0, fzs + aoff[0], fws + aoff[0], invG, invG * L.cw[s]);
    }
    const double2 *msrc = spectra + 2 * npairs * G;
    if (N > 1) {
      for (int a = N - 1; a >= 1; --a) {
        LineSet ls = axis_lines(N, g->dims, a, 1);
        const double *facs[1] = {fzs + aoff[a]};
        const double ones[1] = {1.0};
        if (pow2)
          axis_pass_pow2(ctx, ls, a == N - 1 ? msrc : scratch, scratch, facs, ones, 1, st);
        else
          fft_axis(ctx, ls, a == N - 1 ? msrc : scratch, scratch, 1, facs, ones, 1, st, PKDE_PHASE_STEP_FFT);
      }
      msrc = scratch;
    }
    if (pow2)
      means_pass_pow2(ctx, n1, msrc, rows, fzs + aoff[0], invG, wel, G, (int)B, L.vscale[s], L.dlogt[s], L.eps,
                      L.steps_low, L.steps_over, cs, (int)s, st);
    else
      launch_means(msrc, fzs + aoff[0], invG, s);
  }
  {
    ::pkde::Trace _tr(ctx, PKDE_PHASE_OTHER, st);
    replace_nans_kernel<<<blocks_for(ctx, G), kThreads, 0, st>>>(G, cs, (int)L.S);
  }
  PKDE_CHECK_LAUNCH();
  if (d_density) PKDE_CUDA_TRY(cudaMemcpyAsync(d_density, cs.density, sizeof(double) * G, cudaMemcpyDeviceToDevice, st));
  if (d_selected)
    PKDE_CUDA_TRY(cudaMemcpyAsync(d_selected, cs.selected, sizeof(int32_t) * G, cudaMemcpyDeviceToDevice, st));
}

static void validate_params(const pkde_gradepro_params *p, int64_t n) {
  if (!p) throw invalid("params is NULL");
  grid_validate(&p->grid);
  if (p->n_bootstraps < 2) throw invalid("at least 2 bootstraps are needed (got %d)", p->n_bootstraps);
  if (p->n_steps < 0) throw invalid("n_steps must be non-negative");
  if (n < 2) throw invalid("at least 2 samples are needed");
}

}  // namespace pkde

extern "C" {

int pkde_gradepro_estimate(pkde_ctx *ctx, const pkde_gradepro_params *p, const double *data, int64_t n,
                           const int32_t *boot_idx, uint64_t seed, double *density_out, int32_t *selected_out,
                           uint32_t flags, void *stream) {
  return pkde_guard(ctx, [&] {
    using namespace pkde;
    if (!ctx) throw invalid("context is NULL");
    validate_params(p, n);
    if (!data) throw invalid("data is NULL");
    PKDE_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    const int N = p->grid.ndim;
    const int64_t G = grid_size(&p->grid);
    const bool din = flags & PKDE_DEVICE_INPUT, dout = flags & PKDE_DEVICE_OUTPUT;
    const double *d_data = data;
    if (!din) {
      double *dd = (double *)ensure(ctx, BUF_DATA, sizeof(double) * N * n);
      copy_in(dd, data, sizeof(double) * N * n, false, st);
      d_data = dd;
    }
    const int32_t *d_idx = boot_idx;
    if (boot_idx && !din) {
      int32_t *di = (int32_t *)ensure(ctx, BUF_IDX, sizeof(int32_t) * n * p->n_bootstraps);
      copy_in(di, boot_idx, sizeof(int32_t) * n * p->n_bootstraps, false, st);
      d_idx = di;
    }
    double *dens = density_out;
    int32_t *sel = selected_out;
    if (!dout) {
      char *o = (char *)ensure(ctx, BUF_OUT, (sizeof(double) + sizeof(int32_t)) * G);
      dens = (double *)o;
      sel = (int32_t *)(dens + G);
    }
    Estimation E{p, n, d_data, d_idx, seed};
    run_gradepro(ctx, E, dens, sel, st);
    if (!dout) {
      if (density_out) copy_out(density_out, dens, sizeof(double) * G, false, st);
      if (selected_out) copy_out(selected_out, sel, sizeof(int32_t) * G, false, st);
    }
    PKDE_CUDA_TRY(cudaStreamSynchronize(st));
    collect_trace(ctx);
  });
}

int pkde_set_profiling(pkde_ctx *ctx, int enable) {
  if (!ctx) return PKDE_EINVAL;
  ctx->profiling = enable != 0;
  return PKDE_OK;
}

int pkde_get_stats(pkde_ctx *ctx, pkde_stats *out, int reset) {
  if (!ctx || !out) return PKDE_EINVAL;
  cudaSetDevice(ctx->device);
  cudaDeviceSynchronize();
  pkde::collect_trace(ctx);
  out->launches = ctx->launches;
  for (int i = 0; i < PKDE_NPHASES; ++i) {
    out->phase_launches[i] = ctx->phase_launches[i];
    out->phase_ms[i] = ctx->phase_ms[i];
  }
  if (reset) {
    ctx->launches = 0;
    for (int i = 0; i < PKDE_NPHASES; ++i) {
      ctx->phase_launches[i] = 0;
      ctx->phase_ms[i] = 0.0;
    }
  }
  return PKDE_OK;
}

int pkde_scaled_vmr(pkde_ctx *ctx, int64_t G, int32_t nboot, const double *means, const double *sq, int32_t ndim,
                    const double *t, const double *t0, int64_t n_samples, double *vmr_out, uint32_t flags,
                    void *stream) {
  return pkde_guard(ctx, [&] {
    using namespace pkde;
    if (!ctx) throw invalid("context is NULL");
    if (G < 1 || nboot < 2 || ndim < 1 || ndim > 4 || !means || !sq || !t || !t0 || !vmr_out || n_samples < 1)
      throw invalid("invalid arguments to pkde_scaled_vmr");
    PKDE_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    const bool din = flags & PKDE_DEVICE_INPUT, dout = flags & PKDE_DEVICE_OUTPUT;
    const size_t bytes = sizeof(double2) * G * nboot;
    const double2 *dm = (const double2 *)means, *dv = (const double2 *)sq;
    if (!din) {
      double2 *buf = (double2 *)ensure(ctx, BUF_SCRATCH, 2 * bytes);
      copy_in(buf, means, bytes, false, st);
      copy_in(buf + G * nboot, sq, bytes, false, st);
      dm = buf;
      dv = buf + G * nboot;
    }
    double tmp[4];
    for (int j = 0; j < ndim; ++j) tmp[j] = t[j] * t[j] + t0[j] * t0[j];
    double p = tmp[0];
    for (int j = 1; j < ndim; ++j) p = p * tmp[j];
    const long double n3 = (long double)n_samples * n_samples * n_samples;
    const double scaling = std::pow(p, 1.5) * (double)n3;
    double *out = vmr_out;
    if (!dout) out = (double *)ensure(ctx, BUF_OUT, sizeof(double) * G);
    {
      ::pkde::Trace _tr(ctx, PKDE_PHASE_OTHER, st);
      scaled_vmr_kernel<<<blocks_for(ctx, G), 256, 0, st>>>(G, nboot, dm, dv, (double)n_samples, scaling, out);
    }
    PKDE_CHECK_LAUNCH();
    if (!dout) copy_out(vmr_out, out, sizeof(double) * G, false, st);
    PKDE_CUDA_TRY(cudaStreamSynchronize(st));
  });
}

int pkde_identify_convergence(pkde_ctx *ctx, int64_t G, double *density, const double *means,
                              const double *vmr_current, const double *vmr_prev1, const double *vmr_prev2, double dlogt,
                              double eps, int64_t steps_low, int64_t steps_over, double *minima, uint16_t *counters_low,
                              uint16_t *counters_over, uint8_t *low_density_flags, uint32_t flags, void *stream) {
  return pkde_guard(ctx, [&] {
    using namespace pkde;
    if (!ctx) throw invalid("context is NULL");
    if (G < 1 || !density || !means || !vmr_current || !vmr_prev1 || !vmr_prev2 || !minima || !counters_low ||
        !counters_over || !low_density_flags)
      throw invalid("invalid arguments to pkde_identify_convergence");
    PKDE_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    const bool dev = flags & PKDE_DEVICE_INPUT;
    double *dd = density, *dmin = minima;
    const double *dmu = means, *df = vmr_current, *df1 = vmr_prev1, *df2 = vmr_prev2;
    uint16_t *dcl = counters_low, *dco = counters_over;
    uint8_t *dfl = low_density_flags;
    if (!dev) {
      char *b = (char *)ensure(ctx, BUF_SCRATCH, (sizeof(double) * 6 + 5) * G + 64);
      double *d = (double *)b;
      dd = d;
      double *mu = d + G, *f = d + 2 * G, *f1 = d + 3 * G, *f2 = d + 4 * G;
      dmin = d + 5 * G;
      dcl = (uint16_t *)(d + 6 * G);
      dco = dcl + G;
      dfl = (uint8_t *)(dco + G);
      copy_in(dd, density, sizeof(double) * G, false, st);
      copy_in(mu, means, sizeof(double) * G, false, st);
      copy_in(f, vmr_current, sizeof(double) * G, false, st);
      copy_in(f1, vmr_prev1, sizeof(double) * G, false, st);
      copy_in(f2, vmr_prev2, sizeof(double) * G, false, st);
      copy_in(dmin, minima, sizeof(double) * G, false, st);
      copy_in(dcl, counters_low, sizeof(uint16_t) * G, false, st);
      copy_in(dco, counters_over, sizeof(uint16_t) * G, false, st);
      copy_in(dfl, low_density_flags, G, false, st);
      dmu = mu;
      df = f;
      df1 = f1;
      df2 = f2;
    }
    {
      ::pkde::Trace _tr(ctx, PKDE_PHASE_OTHER, st);
      converge_kernel<<<blocks_for(ctx, G), 256, 0, st>>>(G, dd, dmu, df, df1, df2, dlogt, eps, steps_low, steps_over,
                                                          dmin, dcl, dco, dfl);
    }
    PKDE_CHECK_LAUNCH();
    if (!dev) {
      copy_out(density, dd, sizeof(double) * G, false, st);
      copy_out(minima, dmin, sizeof(double) * G, false, st);
      copy_out(counters_low, dcl, sizeof(uint16_t) * G, false, st);
      copy_out(counters_over, dco, sizeof(uint16_t) * G, false, st);
      copy_out(low_density_flags, dfl, G, false, st);
    }
    PKDE_CUDA_TRY(cudaStreamSynchronize(st));
  });
}

}  // extern "C"
