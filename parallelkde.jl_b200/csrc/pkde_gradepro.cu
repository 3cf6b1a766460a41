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
#include <cstdlib>
#include <cstring>
#include <limits>

#include "pkde_internal.cuh"
#include "pkde_step.cuh"

namespace pkde {

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

// Sums over the samples of one estimation per blockIdx.y: per axis, of x (mean ==
// nullptr) or of (x - mean)^2.  Each of the job's nb blocks writes its partial sums
// (fixed tree order); moments_final_kernel adds a job's partials in order.  The
// partition depends only on the job's own n, so an estimation gets the same sums alone
// and in a batch.
struct MomentJob {
  const double *data;
  int64_t n;
  int ndim;
  int nb;
  double *partial;     // nb x ndim
  const double *mean;  // ndim, or nullptr
  double *out;         // ndim
};

__global__ void moments_partial_kernel(const MomentJob *jobs) {
  __shared__ double sh[32];
  const MomentJob J = jobs[blockIdx.y];
  if ((int)blockIdx.x >= J.nb) return;  // uniform over the block
  for (int j = 0; j < J.ndim; ++j) {
    const double mu = J.mean ? J.mean[j] : 0.0;
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < J.n; i += (int64_t)J.nb * blockDim.x) {
      const double x = J.data[i * J.ndim + j];
      s += J.mean ? (x - mu) * (x - mu) : x;
    }
    const double t = block_sum(s, sh);
    if (threadIdx.x == 0) J.partial[blockIdx.x * J.ndim + j] = t;
  }
}

__global__ void moments_final_kernel(const MomentJob *jobs) {
  const MomentJob J = jobs[blockIdx.x];
  if ((int)threadIdx.x < J.ndim) {
    double s = 0.0;
    for (int b = 0; b < J.nb; ++b) s += J.partial[b * J.ndim + threadIdx.x];
    J.out[threadIdx.x] = s;
  }
}

// The means of the first pass, sum / n with one correctly rounded division per axis (the
// same value the host's division gives), written where the second pass's jobs read them.
__global__ void moments_mean_kernel(const MomentJob *jobs, double *means) {
  const MomentJob J = jobs[blockIdx.x];
  if ((int)threadIdx.x < J.ndim) means[4 * blockIdx.x + threadIdx.x] = __ddiv_rn(J.out[threadIdx.x], (double)J.n);
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

// Per-axis sums of squared deviations from the mean, sum_i (x_ji - mean_j)^2, of several
// sample sets at once (FP64, deterministic): a reduction for the sums, the means on the
// device, a reduction for the squared deviations, and one read-back for the whole set.
// data[e] is N[e] x n[e]; the result goes to centered[4e .. 4e+N[e]-1].
void sample_centered_sums(pkde_ctx *ctx, int count, const double *const *data, const int64_t *n, const int *N,
                          double *centered, cudaStream_t st) {
  if (count < 1) return;
  // jobs[0..count): the sums; jobs[count..2 count): the squared deviations from the means
  std::vector<MomentJob> jobs(2 * (size_t)count);
  int maxnb = 1;
  size_t npart = 0;
  for (int e = 0; e < count; ++e) {
    jobs[e].nb = blocks_for(ctx, n[e]);
    maxnb = std::max(maxnb, jobs[e].nb);
    npart += 4 * (size_t)jobs[e].nb;
  }
  // device: [jobs][sums count x 4][means count x 4][partials]
  const size_t jb = (sizeof(MomentJob) * 2 * count + 255) & ~size_t(255);
  char *m = (char *)ensure(ctx, BUF_MISC, jb + sizeof(double) * (8 * (size_t)count + npart));
  MomentJob *djobs = (MomentJob *)m;
  double *sums = (double *)(m + jb), *means = sums + 4 * count, *partial = means + 4 * count;
  for (int e = 0; e < count; ++e) {
    jobs[e].data = data[e];
    jobs[e].n = n[e];
    jobs[e].ndim = N[e];
    jobs[e].partial = partial;
    partial += 4 * (size_t)jobs[e].nb;
    jobs[e].mean = nullptr;
    jobs[e].out = sums + 4 * e;
    jobs[count + e] = jobs[e];
    jobs[count + e].mean = means + 4 * e;
  }
  PKDE_CUDA_TRY(cudaMemcpyAsync(djobs, jobs.data(), sizeof(MomentJob) * 2 * count, cudaMemcpyHostToDevice, st));
  for (int pass = 0; pass < 2; ++pass) {
    const MomentJob *pj = djobs + (size_t)pass * count;
    {
      ::pkde::Trace _tr(ctx, PKDE_PHASE_OTHER, st);
      moments_partial_kernel<<<dim3((unsigned)maxnb, (unsigned)count), kThreads, 0, st>>>(pj);
    }
    PKDE_CHECK_LAUNCH();
    {
      ::pkde::Trace _tr(ctx, PKDE_PHASE_OTHER, st);
      moments_final_kernel<<<(unsigned)count, 32, 0, st>>>(pj);
    }
    PKDE_CHECK_LAUNCH();
    if (pass == 0) {
      ::pkde::Trace _tr(ctx, PKDE_PHASE_OTHER, st);
      moments_mean_kernel<<<(unsigned)count, 32, 0, st>>>(pj, means);
    }
    if (pass == 0) PKDE_CHECK_LAUNCH();
  }
  std::vector<double> h(4 * (size_t)count);
  PKDE_CUDA_TRY(cudaMemcpyAsync(h.data(), sums, sizeof(double) * 4 * count, cudaMemcpyDeviceToHost, st));
  PKDE_CUDA_TRY(cudaStreamSynchronize(st));
  std::memcpy(centered, h.data(), sizeof(double) * 4 * count);
}

namespace {

// Silverman's rule (DirectSpace.jl:1102-1111) from the FP64 device moments, for several
// estimations at once.  data[e], n[e], N[e] -> bw[4e .. 4e+N[e]-1]
void silverman_batch(pkde_ctx *ctx, int count, const double *const *data, const int64_t *n, const int *N, double *bw,
                     cudaStream_t st) {
  std::vector<double> c(4 * (size_t)std::max(count, 1));
  sample_centered_sums(ctx, count, data, n, N, c.data(), st);
  for (int e = 0; e < count; ++e) {
    const double pref = std::pow(4.0 / ((double)(N[e] + 2) * (double)n[e]), 1.0 / (double)(N[e] + 4));
    for (int j = 0; j < N[e]; ++j) bw[4 * e + j] = pref * std::sqrt(c[4 * e + j] / (double)(n[e] - 1));
  }
}

}  // namespace

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

// The same tables written straight into fz/fw (S x tot each), steps [s0, s1).
// Propagation factor tables of one estimation, computed on the device: for step s and
// grid axis j, fz = exp(-(k t)^2 / 2) and fw = sqrt(fz) over the axis's frequencies k =
// 2 pi fftfreq(n, h) (FourierSpace.jl:228-234 per axis; the full propagator is their
// product over the axes).  Same operation order as the reference's per-axis terms; exp is
// CUDA's, so a factor can differ from a CPU exp in the last bit.
struct TableJob {
  double *fz;            // [S][tot] fz, then [S][tot] fw
  const double *times;   // [S][N]
  int64_t S, tot;
  int N;
  int64_t aoff[5];
  int64_t dims[4];
  double mult[4];        // 2 pi ((1 / h) / n) per axis
};

__global__ void factor_table_kernel(const TableJob *jobs) {
  const TableJob J = jobs[blockIdx.y];
  const int64_t total = J.S * J.tot;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = i / J.tot, r = i - s * J.tot;
    int j = 0;
    while (j + 1 < J.N && r >= J.aoff[j + 1]) ++j;
    const int64_t n = J.dims[j], m = r - J.aoff[j], nneg = (n - 1) / 2 + 1;
    const double mm = (double)(m < nneg ? m : m - n);
    const double kt = __dmul_rn(__dmul_rn(mm, J.mult[j]), J.times[s * J.N + j]);
    const double pv = exp(__dmul_rn(-0.5, __dmul_rn(kt, kt)));
    J.fz[i] = pv;
    J.fz[total + i] = sqrt(pv);
  }
}

static void axis_offsets(const pkde_grid *g, std::vector<int64_t> &axis_off) {
  int64_t tot = 0;
  axis_off.assign(g->ndim + 1, 0);
  for (int j = 0; j < g->ndim; ++j) {
    axis_off[j] = tot;
    tot += g->dims[j];
  }
  axis_off[g->ndim] = tot;
}

// The binning error flags of the call's estimations (after its final synchronisation).
static void check_binning_flags(pkde_ctx *ctx) {
  const int count = ctx->bin_flags_count;
  ctx->bin_flags_count = 0;
  for (int e = 0; e < count; ++e) {
    try {
      binning_flags_check(ctx->bin_flags + 64 * (size_t)e);
    } catch (Error &err) {
      if (count > 1) err.msg = "estimation " + std::to_string(e) + ": " + err.msg;
      ctx->engine_flags_used = 0;  // the call fails on its data; the engine's flags are moot
      throw;
    }
  }
}

// Page-locked staging buffer of the context (grow-only), for asynchronous uploads.
static void *pinned_staging(pkde_ctx *ctx, size_t bytes) {
  if (bytes > ctx->pinned_bytes) {
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    ctx->pinned = nullptr;
    ctx->pinned_bytes = 0;
    PKDE_CUDA_TRY(cudaMallocHost(&ctx->pinned, bytes));
    ctx->pinned_bytes = bytes;
  }
  return ctx->pinned;
}

// One estimation of a call (device pointers).
struct Estimation {
  const pkde_gradepro_params *p;
  int64_t n;
  const double *d_data;
  const int32_t *d_idx;
  uint64_t seed;
  double *d_density;    // may be null
  int32_t *d_selected;  // may be null
};

enum class StepPath { Steps1D, Engine, Generic };

// Everything the device work of one estimation needs.
struct Plan {
  const Estimation *E;
  const pkde_grid *g;
  int N;
  int64_t G, B, npairs;
  StepPath path;
  Ladder L;
  std::vector<int64_t> aoff;
  int64_t tot;
  // device buffers (in the call's arena)
  double2 *spectra;
  ConvState cs;
  double *tables;    // fz tables then fw tables, S x tot each
  double *per_step;  // 1-D: f (S x G), mu (S x G), cw, vscale, dlogt (S each)
  char *bin_scratch;
  int *misc;         // 256-byte block for the binning's flags and max count
  DiracJob job;
};

static size_t al256(size_t x) { return (x + 255) & ~size_t(255); }
static size_t state_bytes(int64_t G) { return al256((sizeof(double) * 5 + sizeof(uint16_t) * 2 + 1 + 4) * G + 256); }

static ConvState bind_state(char *stb, int64_t G) {
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
  return cs;
}

// Bandwidth steps of an N-D estimation on the launch-based path (any axis lengths):
// per step and pair group, inverse FFT passes over axes N..2 then the fused axis-1 pass
// with VMR + Welford, then the means pass with the convergence update.
static void run_generic(pkde_ctx *ctx, Plan &P, cudaStream_t st) {
  const Estimation &E = *P.E;
  const pkde_grid *g = P.g;
  const int N = P.N;
  const int64_t G = P.G;
  const int64_t B = P.B;
  const int64_t npairs = P.npairs;
  const int n1 = (int)g->dims[0];
  const int64_t rows = G / n1;
  const Ladder &L = P.L;
  const std::vector<int64_t> &aoff = P.aoff;
  const int64_t tot = P.tot;
  double2 *spectra = P.spectra;
  ConvState cs = P.cs;
  const double *dfz = P.tables, *dfw = P.tables + L.S * tot;
  const int64_t pair_bytes = (int64_t)sizeof(double2) * 2 * G;
  const int64_t group = std::max<int64_t>(1, std::min<int64_t>(npairs, (48ll << 20) / pair_bytes));
  double2 *scratch = (double2 *)ensure(ctx, BUF_SCRATCH, (size_t)pair_bytes * group);
  double *wel = (double *)ensure(ctx, BUF_WELFORD, sizeof(double) * 2 * G);
  double *wmean = wel, *wm2 = wel + G;
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
    allow_dynamic_smem(ctx, vmr_axis1_kernel<P>, smem);                                                               \
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
    allow_dynamic_smem(ctx, means_converge_kernel<P>, smem);                                                             \
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
}


// The :gradepro estimation of `count` independent sample sets on one stream: each phase
// runs for every estimation before the next phase starts, so the whole call has one
// host synchronisation per phase (Silverman moments, binning read-back), and the
// bandwidth steps of all N-D power-of-two estimations run in one persistent launch.
// An estimation gets the same result alone and in a batch: every kernel partitions its
// work by the estimation's own sizes only.
void run_many(pkde_ctx *ctx, const Estimation *ests, int count, cudaStream_t st) {
  std::vector<Plan> plans(count);
  // ---- Silverman's rule where bw_final is NaN
  std::vector<const double *> sd;
  std::vector<int64_t> sn;
  std::vector<int> sN, who;
  for (int e = 0; e < count; ++e) {
    Plan &P = plans[e];
    P.E = &ests[e];
    P.g = &ests[e].p->grid;
    P.N = P.g->ndim;
    P.G = grid_size(P.g);
    P.B = ests[e].p->n_bootstraps;
    P.npairs = (P.B + 1) / 2;
    bool need = false;
    for (int j = 0; j < P.N; ++j) need |= std::isnan(ests[e].p->bw_final[j]);
    if (need) {
      sd.push_back(ests[e].d_data);
      sn.push_back(ests[e].n);
      sN.push_back(P.N);
      who.push_back(e);
    }
  }
  std::vector<double> sbw(4 * sd.size());
  silverman_batch(ctx, (int)sd.size(), sd.data(), sn.data(), sN.data(), sbw.data(), st);
  // ---- ladders, factor tables, paths
  size_t arena = al256(256 * (size_t)count);  // misc blocks first (one read-back)
  size_t tables_bytes = 0;
  size_t generic_wel = 0, generic_scr = 0;
  std::vector<size_t> off(count);
  for (int e = 0, k = 0; e < count; ++e) {
    Plan &P = plans[e];
    double bw[4];
    const bool need = k < (int)who.size() && who[k] == e;
    for (int j = 0; j < P.N; ++j) bw[j] = need ? sbw[4 * k + j] : 0.0;
    if (need) ++k;
    for (int j = 0; j < P.N; ++j)
      if (!std::isnan(ests[e].p->bw_final[j])) bw[j] = ests[e].p->bw_final[j];
    P.L = make_ladder(ests[e].p, bw, ests[e].n);
    axis_offsets(P.g, P.aoff);
    P.tot = P.aoff[P.N];
    P.path = steps1d_ok(P.g) ? StepPath::Steps1D : (engine_ok(P.g) ? StepPath::Engine : StepPath::Generic);
    if (ctx->step_path == PKDE_STEPS_PER_STEP_LAUNCH) P.path = StepPath::Generic;
    tables_bytes += al256(sizeof(double) * 2 * P.L.S * P.tot);
  }
  // arena: [misc blocks][tables of every estimation][per estimation: spectra, state,
  // 1-D per-step arrays, binning scratch]
  const size_t off_tables = arena;
  arena += tables_bytes;
  size_t times_doubles = 0;
  for (int e = 0; e < count; ++e) times_doubles += (size_t)plans[e].L.S * plans[e].N;
  const size_t tjob_bytes = al256(sizeof(TableJob) * count) + al256(sizeof(double) * times_doubles);
  const size_t off_tjobs = arena;
  arena += tjob_bytes;
  for (int e = 0; e < count; ++e) {
    Plan &P = plans[e];
    off[e] = arena;
    arena += al256(sizeof(double2) * (2 * P.npairs + 1) * P.G);
    arena += state_bytes(P.G);
    if (P.path == StepPath::Steps1D) arena += al256(sizeof(double) * (2 * P.L.S * P.G + 3 * P.L.S));
    arena += dirac_job_scratch(P.g, ests[e].n, P.B);
    if (P.path == StepPath::Generic) {
      generic_wel = std::max(generic_wel, sizeof(double) * 2 * (size_t)P.G);
      const int64_t pair_bytes = (int64_t)sizeof(double2) * 2 * P.G;
      const int64_t group = std::max<int64_t>(1, std::min<int64_t>(P.npairs, (48ll << 20) / pair_bytes));
      generic_scr = std::max(generic_scr, (size_t)(pair_bytes * group));
    }
  }
  char *base = (char *)ensure(ctx, BUF_BATCH, arena);
  if (generic_scr) {  // sized once, so that no buffer grows while kernels are queued
    ensure(ctx, BUF_SCRATCH, generic_scr);
    ensure(ctx, BUF_WELFORD, generic_wel);
  }
  std::vector<size_t> toffs(count);
  size_t toff = 0;
  for (int e = 0; e < count; ++e) {
    Plan &P = plans[e];
    const int64_t S = P.L.S;
    P.misc = (int *)(base + 256 * (size_t)e);
    P.tables = (double *)(base + off_tables + toff);
    toffs[e] = toff;
    toff += al256(sizeof(double) * 2 * S * P.tot);
    char *q = base + off[e];
    P.spectra = (double2 *)q;
    q += al256(sizeof(double2) * (2 * P.npairs + 1) * P.G);
    P.cs = bind_state(q, P.G);
    q += state_bytes(P.G);
    P.per_step = nullptr;
    if (P.path == StepPath::Steps1D) {
      P.per_step = (double *)q;
      q += al256(sizeof(double) * (2 * S * P.G + 3 * S));
    }
    P.bin_scratch = q;
    P.job.g = P.g;
    P.job.d_data = ests[e].d_data;
    P.job.n = ests[e].n;
    P.job.d_idx = ests[e].d_idx;
    P.job.nboot = P.B;
    P.job.seed = ests[e].seed;
    P.job.paired_out = P.spectra;
    dirac_job_bind(P.job, P.bin_scratch, P.misc);
  }
  // ---- binning: phase A for all (queued first, so that the host work below overlaps it)
  for (int e = 0; e < count; ++e) dirac_job_phase_a(ctx, plans[e].job, st);
  // ---- propagation factor tables, on the device: the ladders' times and the job
  // descriptors go up in one copy from page-locked memory, one kernel fills every table
  char *hp = (char *)pinned_staging(ctx, al256(tjob_bytes) + 256 * (size_t)count);
  if (tables_bytes) {
    TableJob *hj = (TableJob *)hp;
    double *ht = (double *)(hp + al256(sizeof(TableJob) * count));
    const double *dt = (const double *)(base + off_tjobs + al256(sizeof(TableJob) * count));
    const double two_pi = 6.283185307179586;
    int64_t tpos = 0, maxtotal = 1;
    for (int e = 0; e < count; ++e) {
      const Plan &P = plans[e];
      TableJob &J = hj[e];
      J.fz = P.tables;
      J.S = P.L.S;
      J.tot = P.tot;
      J.N = P.N;
      for (int q = 0; q <= P.N; ++q) J.aoff[q] = P.aoff[q];
      for (int q = 0; q < P.N; ++q) {
        J.dims[q] = P.g->dims[q];
        J.mult[q] = two_pi * ((1.0 / P.g->h[q]) / (double)P.g->dims[q]);
      }
      std::memcpy(ht + tpos, P.L.times.data(), sizeof(double) * P.L.S * P.N);
      J.times = dt + tpos;
      tpos += P.L.S * P.N;
      maxtotal = std::max<int64_t>(maxtotal, P.L.S * P.tot);
    }
    PKDE_CUDA_TRY(cudaMemcpyAsync(base + off_tjobs, hp, tjob_bytes, cudaMemcpyHostToDevice, st));
    {
      ::pkde::Trace _tr(ctx, PKDE_PHASE_OTHER, st);
      const unsigned bx = (unsigned)std::min<int64_t>((maxtotal + kThreads - 1) / kThreads, (int64_t)ctx->sm_count * 4);
      factor_table_kernel<<<dim3(bx, (unsigned)count), kThreads, 0, st>>>((const TableJob *)(base + off_tjobs));
    }
    PKDE_CHECK_LAUNCH();
  }
  // the binning error flags come back with the call's final synchronisation (invalid data
  // is reported then; what runs on it meanwhile stays in bounds: such samples bin to cell 0)
  int *hflags = (int *)(hp + al256(tjob_bytes));
  PKDE_CUDA_TRY(cudaMemcpyAsync(hflags, base, 256 * (size_t)count, cudaMemcpyDeviceToHost, st));
  ctx->bin_flags = hflags;
  ctx->bin_flags_count = count;
  for (int e = 0; e < count; ++e) dirac_job_phase_b(ctx, plans[e].job, nullptr, st);
  fault_point(ctx, PKDE_FAULT_AFTER_BINNING);
  // ---- forward FFT of every array
  for (int e = 0; e < count; ++e)
    fft_nd(ctx, plans[e].N, plans[e].g->dims, plans[e].spectra, 2 * plans[e].npairs + 1, -1, st,
           PKDE_PHASE_FORWARD_FFT);
  // ---- bandwidth steps
  std::vector<EngineArgs> eng;
  for (int e = 0; e < count; ++e) {
    Plan &P = plans[e];
    const Ladder &L = P.L;
    const int64_t S = L.S;
    const double *dfz = P.tables, *dfw = P.tables + S * P.tot;
    if (P.path == StepPath::Steps1D) {
      // 1-D: every bandwidth step in parallel (one CTA each), then the convergence
      // state machine over the stored per-step f_s and means.
      double *f_all = P.per_step, *mu_all = P.per_step + S * P.G;
      double *d_cw = mu_all + S * P.G, *d_vs = d_cw + S, *d_dl = d_vs + S;
      PKDE_CUDA_TRY(cudaMemcpyAsync(d_cw, L.cw.data(), sizeof(double) * S, cudaMemcpyHostToDevice, st));
      PKDE_CUDA_TRY(cudaMemcpyAsync(d_vs, L.vscale.data(), sizeof(double) * S, cudaMemcpyHostToDevice, st));
      PKDE_CUDA_TRY(cudaMemcpyAsync(d_dl, L.dlogt.data(), sizeof(double) * S, cudaMemcpyHostToDevice, st));
      steps1d(ctx, (int)P.g->dims[0], P.spectra, (int)P.npairs, (int)P.B, (int)S, dfz, dfw, P.tot, d_cw,
              1.0 / (double)P.G, 1.0 / (double)ests[e].n, d_vs, f_all, mu_all, st);
      converge_steps(ctx, P.G, (int)S, f_all, mu_all, d_dl, L.eps, L.steps_low, L.steps_over, P.cs, st);
      continue;
    }
    auto init_state = [&] {
      {
        ::pkde::Trace _tr(ctx, PKDE_PHASE_OTHER, st);
        init_state_kernel<<<blocks_for(ctx, P.G), kThreads, 0, st>>>(P.G, P.cs);
      }
      PKDE_CHECK_LAUNCH();
    };
    if (P.path == StepPath::Generic) {
      init_state();
      run_generic(ctx, P, st);
      continue;
    }
    // N-D: the persistent step engine, schedule parameters per shape (autotuned once)
    EngineArgs A{};
    A.grid = P.g;
    A.npairs = (int)P.npairs;
    A.nboot = (int)P.B;
    A.S = (int)S;
    A.spectra = P.spectra;
    A.fz = dfz;
    A.fw = dfw;
    A.tab_stride = P.tot;
    for (int j = 0; j < P.N; ++j) A.aoff[j] = P.aoff[j];
    A.cw = L.cw.data();
    A.vscale = L.vscale.data();
    A.dlogt = L.dlogt.data();
    A.inv_n = 1.0 / (double)ests[e].n;
    A.eps = L.eps;
    A.steps_low = L.steps_low;
    A.steps_over = L.steps_over;
    A.cs = P.cs;
    autotune_engine(ctx, A, st);  // trial runs (if any) overwrite the state: initialise after
    init_state();
    eng.push_back(A);
  }
  // two persistent launches: estimations whose axes all take the register power-of-two
  // tiles run in the lean kernel instantiation, the others in the one with the
  // mixed-radix and shared-memory tiles (more registers spilled)
  {
    std::vector<EngineArgs> lean, wide;
    for (const EngineArgs &A : eng) (engine_register_only(A.grid) ? lean : wide).push_back(A);
    // Schedules are tuned per shape, one estimation at a time, and the tuned ring slots of
    // many estimations together can exceed the free memory.  The estimations are then
    // packed, in call order, into consecutive launches whose rings fit half of it, each
    // keeping its tuned schedule; only an estimation whose ring alone exceeds that runs
    // with narrow slots (the schedule changes time, never results).  Narrowing every slot
    // of a single launch instead cost the batched mix of 256 estimations more than the
    // launch boundaries do (it ran slower than the same estimations one call each).
    auto launch_fitting = [&](std::vector<EngineArgs> &v) {
      if (v.empty()) return;
      size_t freeb = 0, totalb = 0;
      PKDE_CUDA_TRY(cudaMemGetInfo(&freeb, &totalb));
      size_t budget = (freeb + ctx->buf[BUF_ENGINE].bytes) / 2;
      // PKDE_RING_BUDGET_MB caps the budget (tests use it to force one launch per estimation)
      if (const char *cap = getenv("PKDE_RING_BUDGET_MB"); cap && *cap)
        budget = std::min(budget, (size_t)std::max(0LL, atoll(cap)) << 20);
      size_t i = 0;
      while (i < v.size()) {
        size_t need = 0, j = i;
        for (; j < v.size(); ++j) {
          if (engine_ring_bytes(v[j]) > budget && v[j].tune_slot_mb > kNarrowSlotMB) v[j].tune_slot_mb = kNarrowSlotMB;
          const size_t r = engine_ring_bytes(v[j]);
          if (j > i && need + r > budget) break;
          need += r;
        }
        run_engine_batch(ctx, v.data() + i, (int)(j - i), st);
        i = j;
      }
    };
    launch_fitting(lean);
    launch_fitting(wide);
  }
  // ---- replace_nans! and outputs
  for (int e = 0; e < count; ++e) {
    Plan &P = plans[e];
    if (P.path != StepPath::Steps1D) {
      ::pkde::Trace _tr(ctx, PKDE_PHASE_OTHER, st);
      replace_nans_kernel<<<blocks_for(ctx, P.G), kThreads, 0, st>>>(P.G, P.cs, (int)P.L.S);
    }
    PKDE_CHECK_LAUNCH();
    if (ests[e].d_density)
      PKDE_CUDA_TRY(cudaMemcpyAsync(ests[e].d_density, P.cs.density, sizeof(double) * P.G, cudaMemcpyDeviceToDevice, st));
    if (ests[e].d_selected)
      PKDE_CUDA_TRY(
          cudaMemcpyAsync(ests[e].d_selected, P.cs.selected, sizeof(int32_t) * P.G, cudaMemcpyDeviceToDevice, st));
  }
}

void validate_gradepro_params(const pkde_gradepro_params *p, int64_t n) {
  if (!p) throw invalid("params is NULL");
  grid_validate(&p->grid);
  if (p->n_bootstraps < 2) throw invalid("at least 2 bootstraps are needed (got %d)", p->n_bootstraps);
  if (p->n_steps < 0) throw invalid("n_steps must be non-negative");
  if (n < 2) throw invalid("at least 2 samples are needed");
}

// ------------------------------------------------------------------- :rot estimator
// RoTEstimator.jl: the density is |ifft(P(k, t) * fft(dirac))| with one propagation by
// t = rule-of-thumb time - h/2 (:64-66).  Binning of every sample once (means only,
// :143-148 -> DirectSpace.jl:97-145), unnormalised forward FFT (:148), propagation with
// the per-axis factors exp(-0.5 (k_j t_j)^2) applied on load of the inverse-FFT passes
// (FourierSpace.jl:242-262 split per axis), inverse FFT scaled by 1/G (:203-230), |.|
// (copy_density!, :233-265).
namespace {
__global__ void abs_kernel(int64_t G, const double2 *__restrict__ z, double *__restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < G; i += (int64_t)gridDim.x * blockDim.x) {
    const double2 v = z[i];
    out[i] = sqrt(v.x * v.x + v.y * v.y);
  }
}
}  // namespace

void run_rot(pkde_ctx *ctx, const pkde_grid *g, int rule, const double *d_data, int64_t n, double *d_density,
             cudaStream_t st) {
  const int N = g->ndim;
  const int64_t G = grid_size(g);
  // propagation_time (RoTEstimator.jl:24-49): factor * sqrt(diag(cov(data))), cov with
  // divisor n - 1
  double c[4];
  int Nn = N;
  sample_centered_sums(ctx, 1, &d_data, &n, &Nn, c, st);
  const double factor = rule == PKDE_ROT_SILVERMAN
                            ? std::pow((double)(n * (int64_t)(N + 2)) / 4.0, -1.0 / (double)(N + 4))
                            : std::pow((double)n, -1.0 / (double)(N + 4));
  Ladder L{};
  L.ndim = N;
  L.S = 1;
  L.times.resize(N);
  for (int j = 0; j < N; ++j) L.times[j] = factor * std::sqrt(c[j] / (double)(n - 1)) - g->h[j] / 2;
  std::vector<double> fz, fw;
  std::vector<int64_t> aoff;
  factor_tables(g, L, fz, fw, aoff);
  const int64_t tot = aoff[N];
  // device: [misc block][factor tables][spectrum][binning scratch]
  const size_t off_tab = 256, off_spec = off_tab + al256(sizeof(double) * tot),
               off_scr = off_spec + al256(sizeof(double2) * G);
  char *base = (char *)ensure(ctx, BUF_BATCH, off_scr + dirac_job_scratch(g, n, 0));
  double *tables = (double *)(base + off_tab);
  double2 *spec = (double2 *)(base + off_spec);
  PKDE_CUDA_TRY(cudaMemcpyAsync(tables, fz.data(), sizeof(double) * tot, cudaMemcpyHostToDevice, st));
  DiracJob j;
  j.g = g;
  j.d_data = d_data;
  j.n = n;
  j.nboot = 0;
  j.paired_out = spec;
  dirac_job_bind(j, base + off_scr, (int *)base);
  dirac_job_phase_a(ctx, j, st);
  int h[64];
  PKDE_CUDA_TRY(cudaMemcpyAsync(h, base, 256, cudaMemcpyDeviceToHost, st));
  PKDE_CUDA_TRY(cudaStreamSynchronize(st));
  dirac_job_phase_b(ctx, j, h, st);
  fft_nd(ctx, N, g->dims, spec, 1, -1, st, PKDE_PHASE_FORWARD_FFT);
  for (int a = 0; a < N; ++a) {
    LineSet ls = axis_lines(N, g->dims, a, 1);
    const double *fac[1] = {tables + aoff[a]};
    const double sc[1] = {a == 0 ? 1.0 / (double)G : 1.0};
    fft_axis(ctx, ls, spec, spec, 1, fac, sc, 1, st, PKDE_PHASE_STEP_FFT);
  }
  {
    ::pkde::Trace _tr(ctx, PKDE_PHASE_STEP_MEANS, st);
    abs_kernel<<<blocks_for(ctx, G), kThreads, 0, st>>>(G, spec, d_density);
  }
  PKDE_CHECK_LAUNCH();
}

}  // namespace pkde

extern "C" {

int pkde_gradepro_estimate(pkde_ctx *ctx, const pkde_gradepro_params *p, const double *data, int64_t n,
                           const int32_t *boot_idx, uint64_t seed, double *density_out, int32_t *selected_out,
                           uint32_t flags, void *stream) {
  const double *d[1] = {data};
  const int32_t *i[1] = {boot_idx};
  double *o[1] = {density_out};
  int32_t *so[1] = {selected_out};
  return pkde_gradepro_estimate_batch(ctx, 1, p, d, &n, i, &seed, o, so, flags, stream);
}

int pkde_gradepro_estimate_batch(pkde_ctx *ctx, int32_t count, const pkde_gradepro_params *params,
                                 const double *const *data, const int64_t *n, const int32_t *const *boot_idx,
                                 const uint64_t *seeds, double *const *density_out, int32_t *const *selected_out,
                                 uint32_t flags, void *stream) {
  return pkde_guard(ctx, [&] {
    using namespace pkde;
    if (!ctx) throw invalid("context is NULL");
    if (count < 1 || count > 65535) throw invalid("count must be in 1..65535 (got %d)", count);
    if (!params || !data || !n) throw invalid("params, data and n are required");
    for (int e = 0; e < count; ++e) {
      validate_gradepro_params(&params[e], n[e]);
      if (!data[e]) throw invalid("data[%d] is NULL", e);
    }
    PKDE_CUDA_TRY(cudaSetDevice(ctx->device));
    settle_pending(ctx);
    cudaStream_t st = (cudaStream_t)stream;
    DrainOnError drain{ctx, st};
    const bool din = flags & PKDE_DEVICE_INPUT, dout = flags & PKDE_DEVICE_OUTPUT;
    // host inputs: one device buffer for all samples (and one for all indices)
    std::vector<size_t> doff(count), ioff(count), ooff(count);
    size_t dbytes = 0, ibytes = 0, obytes = 0;
    for (int e = 0; e < count; ++e) {
      const int N = params[e].grid.ndim;
      const int64_t G = grid_size(&params[e].grid);
      doff[e] = dbytes;
      dbytes += al256(sizeof(double) * N * n[e]);
      ioff[e] = ibytes;
      if (boot_idx && boot_idx[e]) ibytes += al256(sizeof(int32_t) * n[e] * params[e].n_bootstraps);
      ooff[e] = obytes;
      obytes += al256((sizeof(double) + sizeof(int32_t)) * G);
    }
    char *ddata = din ? nullptr : (char *)ensure(ctx, BUF_DATA, dbytes);
    char *didx = (din || !ibytes) ? nullptr : (char *)ensure(ctx, BUF_IDX, ibytes);
    char *dout_buf = dout ? nullptr : (char *)ensure(ctx, BUF_OUT, obytes);
    std::vector<Estimation> ests(count);
    for (int e = 0; e < count; ++e) {
      const int N = params[e].grid.ndim;
      const int64_t G = grid_size(&params[e].grid);
      Estimation &E = ests[e];
      E.p = &params[e];
      E.n = n[e];
      E.seed = seeds ? seeds[e] : 0;
      E.d_data = data[e];
      if (!din) {
        copy_in(ddata + doff[e], data[e], sizeof(double) * N * n[e], false, st);
        E.d_data = (const double *)(ddata + doff[e]);
      }
      E.d_idx = (boot_idx && boot_idx[e]) ? boot_idx[e] : nullptr;
      if (E.d_idx && !din) {
        copy_in(didx + ioff[e], boot_idx[e], sizeof(int32_t) * n[e] * params[e].n_bootstraps, false, st);
        E.d_idx = (const int32_t *)(didx + ioff[e]);
      }
      double *dens = density_out ? density_out[e] : nullptr;
      int32_t *sel = selected_out ? selected_out[e] : nullptr;
      if (!dout) {
        dens = dens ? (double *)(dout_buf + ooff[e]) : nullptr;
        sel = sel ? (int32_t *)(dout_buf + ooff[e] + sizeof(double) * G) : nullptr;
      }
      E.d_density = dens;
      E.d_selected = sel;
    }
    run_many(ctx, ests.data(), count, st);
    if (!dout) {
      for (int e = 0; e < count; ++e) {
        const int64_t G = grid_size(&params[e].grid);
        if (ests[e].d_density) copy_out(density_out[e], ests[e].d_density, sizeof(double) * G, false, st);
        if (ests[e].d_selected) copy_out(selected_out[e], ests[e].d_selected, sizeof(int32_t) * G, false, st);
      }
    }
    PKDE_CUDA_TRY(cudaStreamSynchronize(st));
    collect_trace(ctx);
    check_binning_flags(ctx);
    check_engine_flags(ctx);
  });
}

int pkde_rot_estimate(pkde_ctx *ctx, const pkde_grid *grid, int32_t rule, const double *data, int64_t n,
                      double *density_out, uint32_t flags, void *stream) {
  return pkde_guard(ctx, [&] {
    using namespace pkde;
    if (!ctx) throw invalid("context is NULL");
    grid_validate(grid);
    if (rule != PKDE_ROT_SCOTT && rule != PKDE_ROT_SILVERMAN) throw invalid("Rule of thumb %d not implemented.", rule);
    if (n < 2) throw invalid("at least 2 samples are needed");
    if (!data || !density_out) throw invalid("data and density_out are required");
    PKDE_CUDA_TRY(cudaSetDevice(ctx->device));
    settle_pending(ctx);
    cudaStream_t st = (cudaStream_t)stream;
    DrainOnError drain{ctx, st};
    const int N = grid->ndim;
    const int64_t G = grid_size(grid);
    const bool din = flags & PKDE_DEVICE_INPUT, dout = flags & PKDE_DEVICE_OUTPUT;
    const double *d_data = data;
    if (!din) {
      double *dd = (double *)ensure(ctx, BUF_DATA, sizeof(double) * N * n);
      copy_in(dd, data, sizeof(double) * N * n, false, st);
      d_data = dd;
    }
    double *dens = dout ? density_out : (double *)ensure(ctx, BUF_OUT, sizeof(double) * G);
    run_rot(ctx, grid, rule, d_data, n, dens, st);
    if (!dout) copy_out(density_out, dens, sizeof(double) * G, false, st);
    PKDE_CUDA_TRY(cudaStreamSynchronize(st));
    collect_trace(ctx);
  });
}

int pkde_set_step_path(pkde_ctx *ctx, int path) {
  if (!ctx) return PKDE_EINVAL;
  if (path != PKDE_STEPS_AUTO && path != PKDE_STEPS_PER_STEP_LAUNCH) {
    pkde::thread_error(ctx) = "step path must be PKDE_STEPS_AUTO or PKDE_STEPS_PER_STEP_LAUNCH";
    return PKDE_EINVAL;
  }
  ctx->step_path = path;
  return PKDE_OK;
}

int pkde_set_autotune(pkde_ctx *ctx, int enable) {
  if (!ctx) return PKDE_EINVAL;
  ctx->autotune = enable != 0;
  return PKDE_OK;
}

int pkde_set_profiling(pkde_ctx *ctx, int enable) {
  if (!ctx) return PKDE_EINVAL;
  if (enable < PKDE_PROFILE_OFF || enable > PKDE_PROFILE_STEPS) return PKDE_EINVAL;
  ctx->profiling = enable;
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
    settle_pending(ctx);
    cudaStream_t st = (cudaStream_t)stream;
    DrainOnError drain{ctx, st};
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
    settle_pending(ctx);
    cudaStream_t st = (cudaStream_t)stream;
    DrainOnError drain{ctx, st};
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
