// Per-bandwidth-step kernels on power-of-two grid axes (16..4096 points), built on the
// register-resident tile FFT (pkde_regfft.cuh):
//   axis_pass_pow2 : inverse FFT along one axis >= 2 of a batch of arrays, the axis's
//                    propagation factor applied on load (FourierSpace.jl:215-241 split
//                    per axis: the Gaussian propagator is separable);
//   vmr_pass_pow2  : inverse FFT along axis 1 of the bootstrap pairs of a group, then the
//                    variance-to-mean ratio of every bootstrap and its running variance
//                    over bootstraps (DirectSpace.jl:526-584);
//   means_pass_pow2: inverse FFT along axis 1 of the full-sample means, the scaled log
//                    variance and the convergence update (DirectSpace.jl:747-764,
//                    975-1031; GradeProEstimator.jl:638-669).
#include "pkde_regfft.cuh"
#include "pkde_step.cuh"

namespace pkde {
namespace {

// Twiddle tables live in shared memory up to N = 2048.
template <int LOGN>
constexpr bool kTwInSmem = LOGN <= 11;

template <int LOGN>
size_t tile_smem_bytes() {
  using P = Pow2<LOGN>;
  return sizeof(double2) * ((size_t)P::TILE + (kTwInSmem<LOGN> ? P::TWSIZE : 0));
}

template <int LOGN>
__device__ __forceinline__ const double2 *stage_twiddles(double2 *sm_tw, const double2 *__restrict__ tw_g) {
  if constexpr (kTwInSmem<LOGN>) {
    for (int i = threadIdx.x; i < Pow2<LOGN>::TWSIZE; i += blockDim.x) sm_tw[i] = tw_g[i];
    return sm_tw;
  } else {
    return tw_g;
  }
}

// Inverse FFT of NL adjacent lines along axis a >= 2 (lines differ in the inner index).
template <int LOGN>
__global__ void __launch_bounds__(Pow2<LOGN>::THREADS) axis_pass_pow2_kernel(
    const double2 *in, double2 *out, LineSet ls, const double2 *__restrict__ tw_g, const double *__restrict__ f0,
    const double *__restrict__ f1, double s0, double s1, int nfac) {
  using P = Pow2<LOGN>;
  using I = TileIdx<LOGN, true>;
  extern __shared__ double2 smem[];
  double2 *tile = smem;
  const double2 *tw = stage_twiddles<LOGN>(smem + P::TILE, tw_g);
  const int64_t L = (int64_t)blockIdx.x * P::NL + I::line();
  const int t = I::bfly();
  const int64_t base = ls.base(L);
  const int64_t a = L / (ls.inner * ls.outer);
  const bool second = nfac == 2 && (a & 1);
  const double *f = nfac ? (second ? f1 : f0) : nullptr;
  const double sc = nfac ? (second ? s1 : s0) : 1.0;
  double2 v[8];
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int k = in_pos<LOGN>(t, r);
    v[r] = cscale(in[base + (int64_t)k * ls.inner], f ? sc * f[k] : sc);
  }
  __syncthreads();  // twiddles staged
  tile_fft_reg<LOGN, 1, true>(tile, v, tw);
#pragma unroll
  for (int i = 0; i < 8; ++i) out[base + (int64_t)out_pos<LOGN>(t, i) * ls.inner] = v[i];
}

// m = |M|/n, v = |V|/n - m^2, r = v/m (DirectSpace.jl:550-552; 1/n as a product).
__device__ __forceinline__ double vmr_of(double Mv, double Vv, double inv_n) {
  const double m = fabs(Mv) * inv_n;
  const double v = fabs(Vv) * inv_n - m * m;
  return div_nr(v, m);
}

// Welford update of bootstrap i = b + 1 (DirectSpace.jl:572-577), inv = 1/i.
__device__ __forceinline__ void welford(double x, double inv, double &mean, double &m2) {
  const double delta = x - mean;
  mean = fma(delta, inv, mean);
  m2 = fma(delta, x - mean, m2);
}

template <int LOGN>
__global__ void __launch_bounds__(Pow2<LOGN>::THREADS, 2) vmr_pass_pow2_kernel(
    const double2 *__restrict__ in, int npairs, int b0, int nboot, const double2 *__restrict__ tw_g,
    const double *__restrict__ fz, const double *__restrict__ fw, double cz, double cw, double inv_n, int64_t G,
    double *__restrict__ wstate, int first) {
  using P = Pow2<LOGN>;
  using I = TileIdx<LOGN, false>;
  extern __shared__ double2 smem[];
  double2 *tile = smem;
  const double2 *tw = stage_twiddles<LOGN>(smem + P::TILE, tw_g);
  // running (mean, m2) of the thread's 8 points, in shared memory: [i][thread]
  double2 *state = smem + P::TILE + (kTwInSmem<LOGN> ? P::TWSIZE : 0);
  const int64_t row = (int64_t)blockIdx.x * P::NL + I::line();
  const int t = I::bfly();
  const int64_t rbase = row * P::N;
  double *wmean = wstate, *wm2 = wstate + G;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int64_t gi = rbase + out_pos<LOGN>(t, i);
    state[i * P::THREADS + threadIdx.x] = first ? make_double2(0.0, 0.0) : make_double2(wmean[gi], wm2[gi]);
  }
  __syncthreads();  // twiddles staged
  for (int p = 0; p < npairs; ++p) {
    const double2 *zs = in + (int64_t)(2 * p) * G + rbase;
    const double2 *ws = zs + G;
    double2 z[8], w[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int k = in_pos<LOGN>(t, r);
      z[r] = cscale(zs[k], cz * fz[k]);
    }
    tile_fft_reg<LOGN, 1, false>(tile, z, tw);
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int k = in_pos<LOGN>(t, r);
      w[r] = cscale(ws[k], cw * fw[k]);
    }
    tile_fft_reg<LOGN, 1, false>(tile, w, tw);
    const int b = b0 + 2 * p;
    const double inv_a = 1.0 / (double)(b + 1), inv_b = 1.0 / (double)(b + 2);
    const bool has_b = b + 1 < nboot;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      double2 s = state[i * P::THREADS + threadIdx.x];
      welford(vmr_of(z[i].x, w[i].x, inv_n), inv_a, s.x, s.y);
      if (has_b) welford(vmr_of(z[i].y, w[i].y, inv_n), inv_b, s.x, s.y);
      state[i * P::THREADS + threadIdx.x] = s;
    }
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int64_t gi = rbase + out_pos<LOGN>(t, i);
    const double2 s = state[i * P::THREADS + threadIdx.x];
    wmean[gi] = s.x;
    wm2[gi] = s.y;
  }
}

template <int LOGN>
__global__ void __launch_bounds__(Pow2<LOGN>::THREADS) means_pass_pow2_kernel(
    const double2 *__restrict__ in, const double2 *__restrict__ tw_g, const double *__restrict__ fz, double cz,
    const double *__restrict__ wstate, int64_t G, int nboot, double vscale, double dlogt, double eps, int64_t steps_low,
    int64_t steps_over, StepState cs, int step) {
  using P = Pow2<LOGN>;
  using I = TileIdx<LOGN, false>;
  extern __shared__ double2 smem[];
  double2 *tile = smem;
  const double2 *tw = stage_twiddles<LOGN>(smem + P::TILE, tw_g);
  const int64_t row = (int64_t)blockIdx.x * P::NL + I::line();
  const int t = I::bfly();
  const int64_t rbase = row * P::N;
  double2 z[8];
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int k = in_pos<LOGN>(t, r);
    z[r] = cscale(in[rbase + k], cz * fz[k]);
  }
  __syncthreads();  // twiddles staged
  tile_fft_reg<LOGN, 1, false>(tile, z, tw);
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int64_t gi = rbase + out_pos<LOGN>(t, i);
    const double mu = sqrt(z[i].x * z[i].x + z[i].y * z[i].y);
    const double m2 = wstate[G + gi];
    step_update(cs, gi, mu, vscale * m2 / (double)(nboot - 1), dlogt, eps, steps_low, steps_over, step);
  }
}

// 1-D grids: one CTA per bandwidth step, the whole line in one tile.  The CTA runs every
// bootstrap pair (inverse FFT of z and w, VMR, Welford in bootstrap order) and the
// full-sample means, and stores the step's log scaled variance f_s and means mu_s; the
// convergence state machine then runs over the steps (converge_steps_kernel).
template <int LOGN>
__global__ void __launch_bounds__(Pow2<LOGN, 1>::THREADS) steps1d_kernel(
    const double2 *__restrict__ spectra, int npairs, int nboot, const double *__restrict__ fz_all,
    const double *__restrict__ fw_all, int64_t tab_stride, const double *__restrict__ cw, double invG, double inv_n,
    const double *__restrict__ vscale, const double2 *__restrict__ tw_g, double *__restrict__ f_out,
    double *__restrict__ mu_out) {
  using P = Pow2<LOGN, 1>;
  using I = TileIdx<LOGN, false, 1>;
  extern __shared__ double2 smem[];
  double2 *tile = smem;
  double2 *sm_tw = smem + P::TILE;
  for (int i = threadIdx.x; i < P::TWSIZE; i += blockDim.x) sm_tw[i] = tw_g[i];
  const int s = blockIdx.x;
  const double *fz = fz_all + (int64_t)s * tab_stride;
  const double *fw = fw_all + (int64_t)s * tab_stride;
  const double cz_s = invG, cw_s = invG * cw[s];
  const int t = I::bfly();
  double mean[8], m2[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) mean[i] = m2[i] = 0.0;
  __syncthreads();
  for (int p = 0; p < npairs; ++p) {
    const double2 *zs = spectra + (int64_t)(2 * p) * P::N;
    const double2 *ws = zs + P::N;
    double2 z[8], w[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int k = in_pos<LOGN>(t, r);
      z[r] = cscale(zs[k], cz_s * fz[k]);
    }
    tile_fft_reg<LOGN, 1, false, 1>(tile, z, sm_tw);
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int k = in_pos<LOGN>(t, r);
      w[r] = cscale(ws[k], cw_s * fw[k]);
    }
    tile_fft_reg<LOGN, 1, false, 1>(tile, w, sm_tw);
    const int b = 2 * p;
    const double inv_a = 1.0 / (double)(b + 1), inv_b = 1.0 / (double)(b + 2);
    const bool has_b = b + 1 < nboot;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      welford(vmr_of(z[i].x, w[i].x, inv_n), inv_a, mean[i], m2[i]);
      if (has_b) welford(vmr_of(z[i].y, w[i].y, inv_n), inv_b, mean[i], m2[i]);
    }
  }
  const double2 *zf = spectra + (int64_t)(2 * npairs) * P::N;
  double2 z[8];
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int k = in_pos<LOGN>(t, r);
    z[r] = cscale(zf[k], cz_s * fz[k]);
  }
  tile_fft_reg<LOGN, 1, false, 1>(tile, z, sm_tw);
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int x = out_pos<LOGN>(t, i);
    const double v = vscale[s] * m2[i] / (double)(nboot - 1);
    f_out[(int64_t)s * P::N + x] = isfinite(v) ? log(v) : nan("");
    mu_out[(int64_t)s * P::N + x] = sqrt(z[i].x * z[i].x + z[i].y * z[i].y);
  }
}

}  // namespace

const double2 *stage_twiddles_device(pkde_ctx *ctx, int logn) {
  const int key = -logn;  // negative keys: per-stage tables (positive: plain tables)
  auto it = ctx->twiddles.find(key);
  if (it != ctx->twiddles.end()) return it->second.as<double2>();
  std::vector<double2> tw = make_stage_twiddles(logn);
  if (tw.empty()) tw.push_back(make_double2(1.0, 0.0));
  DevBuf &b = ctx->twiddles[key];
  b.ensure(sizeof(double2) * tw.size());
  PKDE_CUDA_TRY(cudaMemcpy(b.ptr, tw.data(), sizeof(double2) * tw.size(), cudaMemcpyHostToDevice));
  return b.as<double2>();
}

namespace {

template <int LOGN>
void launch_axis(pkde_ctx *ctx, const LineSet &ls, const double2 *in, double2 *out, const double *const *factors,
                 const double *scal, int nfac, cudaStream_t st) {
  using P = Pow2<LOGN>;
  const size_t smem = tile_smem_bytes<LOGN>();
  allow_dynamic_smem(ctx, axis_pass_pow2_kernel<LOGN>, smem);
  const double2 *tw = stage_twiddles_device(ctx, LOGN);
  const int64_t blocks = ls.nlines() / P::NL;
  {
    Trace tr(ctx, PKDE_PHASE_STEP_FFT, st);
    axis_pass_pow2_kernel<LOGN><<<(unsigned)blocks, P::THREADS, smem, st>>>(
        in, out, ls, tw, factors ? factors[0] : nullptr, (factors && nfac > 1) ? factors[1] : nullptr,
        scal ? scal[0] : 1.0, (scal && nfac > 1) ? scal[1] : 1.0, nfac);
  }
  PKDE_CHECK_LAUNCH();
}

template <int LOGN>
void launch_vmr(pkde_ctx *ctx, const double2 *in, int npairs, int b0, int nboot, int64_t rows, const double *fz,
                const double *fw, double cz, double cw, double inv_n, int64_t G, double *wstate, int first,
                cudaStream_t st) {
  using P = Pow2<LOGN>;
  const size_t smem = tile_smem_bytes<LOGN>() + sizeof(double2) * 8 * P::THREADS;
  allow_dynamic_smem(ctx, vmr_pass_pow2_kernel<LOGN>, smem);
  const double2 *tw = stage_twiddles_device(ctx, LOGN);
  {
    Trace tr(ctx, PKDE_PHASE_STEP_VMR, st);
    vmr_pass_pow2_kernel<LOGN><<<(unsigned)(rows / P::NL), P::THREADS, smem, st>>>(in, npairs, b0, nboot, tw, fz, fw,
                                                                                 cz, cw, inv_n, G, wstate, first);
  }
  PKDE_CHECK_LAUNCH();
}

template <int LOGN>
void launch_means(pkde_ctx *ctx, const double2 *in, int64_t rows, const double *fz, double cz, const double *wstate,
                  int64_t G, int nboot, double vscale, double dlogt, double eps, int64_t steps_low,
                  int64_t steps_over, const StepState &cs, int step, cudaStream_t st) {
  using P = Pow2<LOGN>;
  const size_t smem = tile_smem_bytes<LOGN>();
  allow_dynamic_smem(ctx, means_pass_pow2_kernel<LOGN>, smem);
  const double2 *tw = stage_twiddles_device(ctx, LOGN);
  {
    Trace tr(ctx, PKDE_PHASE_STEP_MEANS, st);
    means_pass_pow2_kernel<LOGN><<<(unsigned)(rows / P::NL), P::THREADS, smem, st>>>(
        in, tw, fz, cz, wstate, G, nboot, vscale, dlogt, eps, steps_low, steps_over, cs, step);
  }
  PKDE_CHECK_LAUNCH();
}

int ilog2_exact(int64_t n) {
  if (n < 16 || n > 4096 || (n & (n - 1))) return -1;
  int l = 0;
  while ((int64_t(1) << l) < n) ++l;
  return l;
}

template <int LOGN>
void launch_steps1d(pkde_ctx *ctx, const double2 *spectra, int npairs, int nboot, int S, const double *fz_all,
                    const double *fw_all, int64_t tab_stride, const double *cw, double invG, double inv_n,
                    const double *vscale, double *f_out, double *mu_out, cudaStream_t st) {
  using P = Pow2<LOGN, 1>;
  const size_t smem = sizeof(double2) * ((size_t)P::TILE + P::TWSIZE);
  allow_dynamic_smem(ctx, steps1d_kernel<LOGN>, smem);
  const double2 *tw = stage_twiddles_device(ctx, LOGN);
  {
    Trace tr(ctx, PKDE_PHASE_STEP_VMR, st);
    steps1d_kernel<LOGN><<<(unsigned)S, P::THREADS, smem, st>>>(spectra, npairs, nboot, fz_all, fw_all, tab_stride, cw,
                                                               invG, inv_n, vscale, tw, f_out, mu_out);
  }
  PKDE_CHECK_LAUNCH();
}

__global__ void converge_steps_kernel(int64_t G, int S, const double *__restrict__ f_all,
                                      const double *__restrict__ mu_all, const double *__restrict__ dlogt, double eps,
                                      int64_t steps_low, int64_t steps_over, StepState cs) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < G; i += (int64_t)gridDim.x * blockDim.x)
    converge_point_all_steps(cs, i, G, S, f_all, mu_all, dlogt, eps, steps_low, steps_over);
}

int lines_per_tile(int logn) { return (1 << logn) / 8 > 256 ? 1 : 256 * 8 / (1 << logn); }

}  // namespace

bool steps1d_ok(const pkde_grid *g) {
  if (g->ndim != 1) return false;
  const int ln = ilog2_exact(g->dims[0]);
  return ln >= 8 && ln <= 12;
}

void steps1d(pkde_ctx *ctx, int n1, const double2 *spectra, int npairs, int nboot, int S, const double *fz_all,
             const double *fw_all, int64_t tab_stride, const double *cw, double invG, double inv_n,
             const double *vscale, double *f_out, double *mu_out, cudaStream_t st) {
#define PKDE_CALL(L) \
  launch_steps1d<L>(ctx, spectra, npairs, nboot, S, fz_all, fw_all, tab_stride, cw, invG, inv_n, vscale, f_out, mu_out, st)
  switch (ilog2_exact(n1)) {
    case 8: PKDE_CALL(8); break;
    case 9: PKDE_CALL(9); break;
    case 10: PKDE_CALL(10); break;
    case 11: PKDE_CALL(11); break;
    case 12: PKDE_CALL(12); break;
    default: throw Error{PKDE_EUNSUPPORTED, "1-D grid length not supported by the step-parallel path"};
  }
#undef PKDE_CALL
}

void converge_steps(pkde_ctx *ctx, int64_t G, int S, const double *f_all, const double *mu_all, const double *dlogt,
                    double eps, int64_t steps_low, int64_t steps_over, const StepState &cs, cudaStream_t st) {
  const int threads = 128;
  const int64_t blocks = std::min<int64_t>((G + threads - 1) / threads, (int64_t)ctx->sm_count * 16);
  {
    Trace tr(ctx, PKDE_PHASE_STEP_MEANS, st);
    converge_steps_kernel<<<(unsigned)blocks, threads, 0, st>>>(G, S, f_all, mu_all, dlogt, eps, steps_low, steps_over,
                                                                cs);
  }
  PKDE_CHECK_LAUNCH();
}

bool pow2_path_ok(const pkde_grid *g) {
  const int64_t G = grid_size(g);
  for (int j = 0; j < g->ndim; ++j) {
    const int ln = ilog2_exact(g->dims[j]);
    if (ln < 0) return false;
    const int64_t lines = G / g->dims[j];
    const int nl = lines_per_tile(ln);
    if (lines % nl) return false;
    // axes >= 2: a tile spans NL adjacent inner indices, which must not straddle
    int64_t inner = 1;
    for (int i = 0; i < j; ++i) inner *= g->dims[i];
    if (j > 0 && inner % nl) return false;
  }
  return true;
}

#define PKDE_POW2_SWITCH(LN, CALL) \
  switch (LN) {                    \
    case 4: CALL(4); break;        \
    case 5: CALL(5); break;        \
    case 6: CALL(6); break;        \
    case 7: CALL(7); break;        \
    case 8: CALL(8); break;        \
    case 9: CALL(9); break;        \
    case 10: CALL(10); break;      \
    case 11: CALL(11); break;      \
    case 12: CALL(12); break;      \
    default: throw Error{PKDE_EUNSUPPORTED, "axis length not supported by the power-of-two path"}; \
  }

void axis_pass_pow2(pkde_ctx *ctx, const LineSet &ls, const double2 *in, double2 *out, const double *const *factors,
                    const double *scal, int nfac, cudaStream_t st) {
#define PKDE_CALL(L) launch_axis<L>(ctx, ls, in, out, factors, scal, nfac, st)
  PKDE_POW2_SWITCH(ilog2_exact(ls.n), PKDE_CALL)
#undef PKDE_CALL
}

void vmr_pass_pow2(pkde_ctx *ctx, int n1, const double2 *in, int npairs, int b0, int nboot, int64_t rows,
                   const double *fz, const double *fw, double cz, double cw, double inv_n, int64_t G, double *wstate,
                   int first, cudaStream_t st) {
#define PKDE_CALL(L) launch_vmr<L>(ctx, in, npairs, b0, nboot, rows, fz, fw, cz, cw, inv_n, G, wstate, first, st)
  PKDE_POW2_SWITCH(ilog2_exact(n1), PKDE_CALL)
#undef PKDE_CALL
}

void means_pass_pow2(pkde_ctx *ctx, int n1, const double2 *in, int64_t rows, const double *fz, double cz,
                     const double *wstate, int64_t G, int nboot, double vscale, double dlogt, double eps,
                     int64_t steps_low, int64_t steps_over, const StepState &cs, int step, cudaStream_t st) {
#define PKDE_CALL(L) \
  launch_means<L>(ctx, in, rows, fz, cz, wstate, G, nboot, vscale, dlogt, eps, steps_low, steps_over, cs, step, st)
  PKDE_POW2_SWITCH(ilog2_exact(n1), PKDE_CALL)
#undef PKDE_CALL
}

}  // namespace pkde
