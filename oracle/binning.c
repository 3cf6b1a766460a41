/*
 * TEST INFRASTRUCTURE ONLY.  FP64 CPU restatement of the reference's Dirac-sequence
 * binning, used by tests/, __graft_entry__.smoke() and bench.py's CPU baseline as the
 * checker.  The product path never links this file.
 *
 * Follows ParallelKDE.jl:
 *   src/StatisticsPropagation/DirectSpace.jl:196-242  generate_dirac_cpu! (mean + squared)
 *   src/StatisticsPropagation/DirectSpace.jl:97-145   initialize_dirac_sequence(::Val{:serial})
 *   src/StatisticsPropagation/DirectSpace.jl:479-498  check_data
 *
 * Semantics reproduced bit for bit:
 *   delta = x - lo;  l = floor(delta / h) (IEEE division);  r_h = rem(delta, h) == fmod;
 *   r_l = h - r_h;  corner bit for axis j (1-based) is (c >> (N - j)) & 1, a set bit
 *   selects the lower cell and the factor r_l, a clear bit the upper cell and r_h;
 *   product = prod(r_l[mask]) * prod(r_h[!mask]) with each prod a left fold
 *   (Julia's mapreduce for short vectors), an empty prod being 1.0;
 *   term = product / (n * prod(h)^2);  M[cell] += term;  V[cell] += term * term,
 *   accumulated sequentially in draw order, one bootstrap column at a time.
 * Compile without -ffast-math and with -ffp-contract=off so that no FMA is formed.
 */
#include <math.h>
#include <stdint.h>
#include <stddef.h>
#include <stdlib.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* Returns 0 on success, 1 if a sample lies on or beyond the grid bounds (the reference
 * throws ArgumentError there), 2 if a sample would address the cell past the last grid
 * point (x within one rounding of the upper bound; the reference writes out of bounds). */
int oracle_check_data(int ndim, const double *lo, const double *hi, const double *h,
                      const int64_t *dims, const double *data, int64_t n) {
  for (int64_t s = 0; s < n; ++s) {
    for (int j = 0; j < ndim; ++j) {
      double x = data[s * ndim + j];
      if ((x >= hi[j]) | (x <= lo[j])) return 1;
      double l = floor((x - lo[j]) / h[j]);
      if (l + 1.0 >= (double)dims[j]) return 2;
    }
  }
  return 0;
}

/* m, v: double sums (ext == 0, the reference's sequential FP64 sums) or long double sums
 * (ext == 1: the same terms accumulated in 80-bit extended precision, later rounded once --
 * a more exact binning, of the kind a fixed-point or compensated accumulation gives; used
 * to tell which grid points' decisions depend on the rounding of the binned sums). */
static void dirac_one(int ndim, const int64_t *dims, const double *lo, const double *h,
                      const double *data, int64_t n, const int32_t *col, void *m, void *v, int ext) {
  double spacing_prod = h[0];
  for (int j = 1; j < ndim; ++j) spacing_prod = spacing_prod * h[j];
  const double spacing_squared = spacing_prod * spacing_prod;
  const double denom = (double)n * spacing_squared;
  int64_t stride[4];
  stride[0] = 1;
  for (int j = 1; j < ndim; ++j) stride[j] = stride[j - 1] * dims[j - 1];

  for (int64_t d = 0; d < n; ++d) {
    const double *x = data + (int64_t)(col[d] - 1) * ndim;
    int64_t il[4];
    double rh[4], rl[4];
    for (int j = 0; j < ndim; ++j) {
      double delta = x[j] - lo[j];
      il[j] = (int64_t)floor(delta / h[j]); /* 0-based lower cell */
      rh[j] = fmod(delta, h[j]);
      rl[j] = h[j] - rh[j];
    }
    const int ncorner = 1 << ndim;
    for (int c = 0; c < ncorner; ++c) {
      double pl = 1.0, ph = 1.0;
      int nl = 0, nh = 0;
      int64_t cell = 0;
      for (int j = 0; j < ndim; ++j) {
        int lower = (c >> (ndim - 1 - j)) & 1;
        if (lower) {
          pl = (nl == 0) ? rl[j] : pl * rl[j];
          ++nl;
          cell += il[j] * stride[j];
        } else {
          ph = (nh == 0) ? rh[j] : ph * rh[j];
          ++nh;
          cell += (il[j] + 1) * stride[j];
        }
      }
      double product = pl * ph;
      double term = product / denom;
      if (ext) {
        ((long double *)m)[cell] += term;
        if (v) ((long double *)v)[cell] += term * term;
      } else {
        ((double *)m)[cell] += term;
        if (v) ((double *)v)[cell] += term * term;
      }
    }
  }
}

/* The same binning with the sums of each bootstrap column accumulated in long double and
 * rounded to FP64 at the end (see DIRAC_ONE). */
int oracle_dirac_ext(int ndim, const int64_t *dims, const double *lo, const double *hi,
                     const double *h, const double *data, int64_t n, const int32_t *idx,
                     int64_t nboot, double *means, double *sq, int nthreads) {
  if (ndim < 1 || ndim > 4) return 3;
  int rc = oracle_check_data(ndim, lo, hi, h, dims, data, n);
  if (rc) return rc;
  int64_t G = 1;
  for (int j = 0; j < ndim; ++j) G *= dims[j];
  for (int64_t b = 0; b < n * nboot; ++b)
    if (idx[b] < 1 || idx[b] > n) return 4;
#ifdef _OPENMP
  if (nthreads < 1) nthreads = 1;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
#endif
  for (int64_t b = 0; b < nboot; ++b) {
    long double *am = (long double *)calloc((size_t)G, sizeof(long double));
    long double *av = sq ? (long double *)calloc((size_t)G, sizeof(long double)) : NULL;
    dirac_one(ndim, dims, lo, h, data, n, idx + b * n, am, av, 1);
    for (int64_t g = 0; g < G; ++g) {
      means[b * G + g] = (double)am[g];
      if (sq) sq[b * G + g] = (double)av[g];
    }
    free(am);
    free(av);
  }
  (void)nthreads;
  return 0;
}

/* means/sq: G x B, column-major (grid axis 1 fastest, bootstrap slowest), zeroed by the
 * caller.  idx: n x B, column-major, 1-based.  sq may be NULL (means-only variant,
 * DirectSpace.jl:243-287).  nthreads > 1 parallelises over bootstrap columns like the
 * reference's :threaded method (DirectSpace.jl:146-194); each column is still
 * accumulated sequentially, so the result does not depend on nthreads. */
int oracle_dirac(int ndim, const int64_t *dims, const double *lo, const double *hi,
                 const double *h, const double *data, int64_t n, const int32_t *idx,
                 int64_t nboot, double *means, double *sq, int nthreads) {
  if (ndim < 1 || ndim > 4) return 3;
  int rc = oracle_check_data(ndim, lo, hi, h, dims, data, n);
  if (rc) return rc;
  int64_t G = 1;
  for (int j = 0; j < ndim; ++j) G *= dims[j];
  for (int64_t b = 0; b < n * nboot; ++b)
    if (idx[b] < 1 || idx[b] > n) return 4;
#ifdef _OPENMP
  if (nthreads < 1) nthreads = 1;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
#endif
  for (int64_t b = 0; b < nboot; ++b) {
    dirac_one(ndim, dims, lo, h, data, n, idx + b * n, means + b * G, sq ? sq + b * G : NULL, 0);
  }
  (void)nthreads;
  return 0;
}
