// Per-grid-point convergence state and the step update shared by the step kernels.
#pragma once

#include "pkde_internal.cuh"

namespace pkde {

// Convergence state of every grid point (DensityState, GradeProEstimator.jl:515-615),
// plus the outputs: density, selected step, and the last step's means.
struct StepState {
  double *f1, *f2, *minima, *density, *mu_last;
  uint16_t *c_low, *c_over;
  uint8_t *flags;
  int32_t *selected;
};

struct StabilityResult {
  bool more_stable;
  double new_min;
  uint16_t c_low, c_over;
  uint8_t flag;
};

// find_stability (DirectSpace.jl:975-1031) with first/second_difference (:1092-1100),
// in FP64.  Explicit-rounding intrinsics keep the operation order of the reference.
__device__ __forceinline__ StabilityResult find_stability(double f, double f1, double f2, double dlogt, double eps,
                                                          int64_t steps_low, int64_t steps_over, double minimum,
                                                          uint16_t c_low, uint16_t c_over, uint8_t flag) {
  const double d1 = log(fabs(__ddiv_rn(__dsub_rn(f, f1), __dmul_rn(2.0, dlogt))));
  const double d2 = log(fabs(__ddiv_rn(__dadd_rn(__dsub_rn(f, __dmul_rn(2.0, f1)), f2), __dmul_rn(dlogt, dlogt))));
  StabilityResult r{false, nan(""), c_low, c_over, flag};
  if (!flag) {
    if (d2 < eps) {
      if (((d1 < minimum) || isnan(minimum)) && ((int64_t)c_over <= steps_over)) {
        r.more_stable = true;
        r.new_min = d1;
        r.c_over = 0;
      } else {
        r.c_over = (uint16_t)(c_over + 1);
      }
    } else {
      r.c_low = (uint16_t)(c_low + 1);
      if ((int64_t)r.c_low > steps_low) {
        r.flag = 1;
        minimum = nan("");
      }
    }
  } else {
    if ((d2 < eps) && isnan(minimum)) {
      r.more_stable = true;
      r.new_min = d1;
    }
  }
  if (isnan(r.new_min)) r.new_min = minimum;
  return r;
}

// One step of update_state! (GradeProEstimator.jl:638-669) at grid point i:
// v = scaled bootstrap variance of the VMR (DirectSpace.jl:579), mu = the means.
// CG = true: the state was written by other CTAs of the same kernel, so it is read
// through L2 (ld.global.cg) and never from a possibly stale L1 line.
template <class T, bool CG>
__device__ __forceinline__ T ld_state(const T *p) {
  if constexpr (CG) return __ldcg(p);
  return *p;
}
template <bool CG = false>
__device__ __forceinline__ void step_update(const StepState &cs, int64_t i, double mu, double v, double dlogt,
                                            double eps, int64_t steps_low, int64_t steps_over, int step) {
  const double f = isfinite(v) ? log(v) : nan("");
  const double f1 = ld_state<double, CG>(cs.f1 + i), f2 = ld_state<double, CG>(cs.f2 + i);
  const uint16_t cl = ld_state<unsigned short, CG>(reinterpret_cast<const unsigned short *>(cs.c_low + i));
  const uint16_t co = ld_state<unsigned short, CG>(reinterpret_cast<const unsigned short *>(cs.c_over + i));
  const uint8_t fl = (uint8_t)ld_state<unsigned char, CG>(reinterpret_cast<const unsigned char *>(cs.flags + i));
  StabilityResult r =
      find_stability(f, f1, f2, dlogt, eps, steps_low, steps_over, ld_state<double, CG>(cs.minima + i), cl, co, fl);
  cs.c_low[i] = r.c_low;
  cs.c_over[i] = r.c_over;
  cs.flags[i] = r.flag;
  cs.minima[i] = r.new_min;
  if (r.more_stable) {
    cs.density[i] = mu;
    cs.selected[i] = step;
  }
  cs.f2[i] = f1;
  cs.f1[i] = f;
  cs.mu_last[i] = mu;
}

// The convergence state machine of one grid point over all steps, from the stored
// per-step log variances f[s*G + i] and means mu[s*G + i]; state kept in registers.
__device__ __forceinline__ void converge_point_all_steps(const StepState &cs, int64_t i, int64_t G, int S,
                                                        const double *f_all, const double *mu_all,
                                                        const double *dlogt, double eps, int64_t steps_low,
                                                        int64_t steps_over) {
  double f1 = nan(""), f2 = nan(""), minimum = nan(""), density = nan(""), mu = nan("");
  uint16_t c_low = 0, c_over = 0;
  uint8_t flag = 0;
  int32_t selected = -1;
  for (int s = 0; s < S; ++s) {
    const double f = f_all[(int64_t)s * G + i];
    mu = mu_all[(int64_t)s * G + i];
    StabilityResult r = find_stability(f, f1, f2, dlogt[s], eps, steps_low, steps_over, minimum, c_low, c_over, flag);
    c_low = r.c_low;
    c_over = r.c_over;
    flag = r.flag;
    minimum = r.new_min;
    if (r.more_stable) {
      density = mu;
      selected = s;
    }
    f2 = f1;
    f1 = f;
  }
  // replace_nans! (GradeProEstimator.jl:1053-1072)
  if (isnan(density)) density = mu;
  cs.density[i] = density;
  cs.selected[i] = selected < 0 ? S : selected;
  cs.mu_last[i] = mu;
  cs.f1[i] = f1;
  cs.f2[i] = f2;
  cs.minima[i] = minimum;
  cs.c_low[i] = c_low;
  cs.c_over[i] = c_over;
  cs.flags[i] = flag;
}

// persistent step engine (pkde_engine.cu)
struct EngineArgs {
  const pkde_grid *grid;
  int npairs, nboot, S;
  const double2 *spectra;
  const double *fz, *fw;  // per-step factor tables [S][tab_stride], axis j at aoff[j]
  int64_t tab_stride;
  int64_t aoff[4];
  const double *cw, *vscale, *dlogt;  // host arrays of S values
  double inv_n, eps;
  int64_t steps_low, steps_over;
  StepState cs;
  // schedule parameters (0: default): ring-slot MB, tiles per axis-pass item, pipeline
  // delay between the passes of a batch
  int tune_slot_mb = 0, tune_tpi = 0, tune_delay = 0, tune_qextra = 0;
};
bool engine_ok(const pkde_grid *g);
// Every axis on the register power-of-two tiles (the engine's lean instantiation).
bool engine_register_only(const pkde_grid *g);
// Per-shape schedule parameters: from the context's cache, else (autotuning on) timed
// trial runs of the estimation's first bandwidth steps.  Overwrites the estimation's
// convergence state (the caller initialises it afterwards).
void autotune_engine(pkde_ctx *ctx, EngineArgs &args, cudaStream_t st);
void run_engine(pkde_ctx *ctx, const EngineArgs &args, cudaStream_t st);
// The error flags of the engine launches queued since the last check: call after the stream
// has synchronised; throws if a launch gave up on a dependency wait.
void check_engine_flags(pkde_ctx *ctx);
// Device bytes of the estimation's ring slots under its schedule parameters.
size_t engine_ring_bytes(const EngineArgs &args);
// Ring slots of at most this size are always allowed; wider ones only within a memory budget.
constexpr int kNarrowSlotMB = 64;
// Several estimations in one persistent launch (their EngineArgs are independent).
void run_engine_batch(pkde_ctx *ctx, const EngineArgs *args, int count, cudaStream_t st);

// power-of-two path (pkde_step.cu)
bool steps1d_ok(const pkde_grid *g);
void steps1d(pkde_ctx *ctx, int n1, const double2 *spectra, int npairs, int nboot, int S, const double *fz_all,
             const double *fw_all, int64_t tab_stride, const double *cw, double invG, double inv_n,
             const double *vscale, double *f_out, double *mu_out, cudaStream_t st);
void converge_steps(pkde_ctx *ctx, int64_t G, int S, const double *f_all, const double *mu_all, const double *dlogt,
                    double eps, int64_t steps_low, int64_t steps_over, const StepState &cs, cudaStream_t st);
bool pow2_path_ok(const pkde_grid *g);
void axis_pass_pow2(pkde_ctx *ctx, const LineSet &ls, const double2 *in, double2 *out, const double *const *factors,
                    const double *scal, int nfac, cudaStream_t st);
void vmr_pass_pow2(pkde_ctx *ctx, int n1, const double2 *in, int npairs, int b0, int nboot, int64_t rows,
                   const double *fz, const double *fw, double cz, double cw, double inv_n, int64_t G, double *wstate,
                   int first, cudaStream_t st);
void means_pass_pow2(pkde_ctx *ctx, int n1, const double2 *in, int64_t rows, const double *fz, double cz,
                     const double *wstate, int64_t G, int nboot, double vscale, double dlogt, double eps,
                     int64_t steps_low, int64_t steps_over, const StepState &cs, int step, cudaStream_t st);

}  // namespace pkde
