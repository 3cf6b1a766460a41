// Grid construction from (device-resident) samples and the normalised density, on the
// device: find_grid (src/Grids/Grids.jl:252-300) and get_density(...; normalize=true)
// (src/ParallelKDE.jl:189-202) without copying the samples or the density to the host.
#include <algorithm>
#include <cstring>

#include "pkde_internal.cuh"

namespace pkde {
namespace {

constexpr int kThreads = 256;

// Per-axis minimum and maximum: per-block results, then one block folds them.  Both
// are exact and order-independent.
__global__ void extrema_partial_kernel(const double *__restrict__ data, int64_t n, int ndim, double *partial) {
  __shared__ double smin[kThreads / 32][4], smax[kThreads / 32][4];
  double lo[4], hi[4];
  for (int j = 0; j < 4; ++j) {
    lo[j] = INFINITY;
    hi[j] = -INFINITY;
  }
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    for (int j = 0; j < ndim; ++j) {
      const double x = data[i * ndim + j];
      lo[j] = fmin(lo[j], x);
      hi[j] = fmax(hi[j], x);
    }
  for (int j = 0; j < ndim; ++j)
    for (int o = 16; o > 0; o >>= 1) {
      lo[j] = fmin(lo[j], __shfl_xor_sync(0xffffffffu, lo[j], o));
      hi[j] = fmax(hi[j], __shfl_xor_sync(0xffffffffu, hi[j], o));
    }
  if ((threadIdx.x & 31) == 0)
    for (int j = 0; j < ndim; ++j) {
      smin[threadIdx.x >> 5][j] = lo[j];
      smax[threadIdx.x >> 5][j] = hi[j];
    }
  __syncthreads();
  if (threadIdx.x < ndim) {
    double a = INFINITY, b = -INFINITY;
    for (int w = 0; w < kThreads / 32; ++w) {
      a = fmin(a, smin[w][threadIdx.x]);
      b = fmax(b, smax[w][threadIdx.x]);
    }
    partial[(int64_t)blockIdx.x * 8 + threadIdx.x] = a;
    partial[(int64_t)blockIdx.x * 8 + 4 + threadIdx.x] = b;
  }
}

__global__ void extrema_final_kernel(const double *partial, int nblocks, int ndim, double *out) {
  if (threadIdx.x < ndim) {
    double a = INFINITY, b = -INFINITY;
    for (int k = 0; k < nblocks; ++k) {
      a = fmin(a, partial[k * 8 + threadIdx.x]);
      b = fmax(b, partial[k * 8 + 4 + threadIdx.x]);
    }
    out[threadIdx.x] = a;
    out[4 + threadIdx.x] = b;
  }
}

// FP64 sum of the density (per-block tree sums in a fixed order), then density /=
// sum * dx.
__global__ void sum_partial_kernel(const double *__restrict__ d, int64_t G, double *partial) {
  __shared__ double sh[kThreads / 32];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < G; i += (int64_t)gridDim.x * blockDim.x)
    s += d[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) t += sh[w];
    partial[blockIdx.x] = t;
  }
}

__global__ void normalize_kernel(double *d, int64_t G, const double *partial, int nblocks, double dx) {
  __shared__ double scale;
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < nblocks; ++k) t += partial[k];
    scale = t * dx;
  }
  __syncthreads();
  const double c = scale;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < G; i += (int64_t)gridDim.x * blockDim.x)
    d[i] = d[i] / c;
}

// Step of range(lo, stop=hi, length=n): (hi - lo)/(n - 1) rounded once.  The
// difference is kept exactly as a double-double (TwoSum), the quotient refined by one
// residual step (exact remainder by fma).
double range_step(double lo, double hi, int64_t n) {
  const double s = hi - lo;
  const double bb = s - hi;
  const double err = (hi - (s - bb)) + (-lo - bb);
  const double m = (double)(n - 1);
  const double q = s / m;
  const double r = std::fma(-q, m, s) + err;
  return q + r / m;
}

}  // namespace
}  // namespace pkde

extern "C" {

int pkde_find_grid(pkde_ctx *ctx, int32_t ndim, const double *data, int64_t n, const int64_t *dims,
                   const double *steps, const double *padding, pkde_grid *out, uint32_t flags, void *stream) {
  return pkde_guard(ctx, [&] {
    using namespace pkde;
    if (!ctx) throw invalid("context is NULL");
    if (ndim < 1 || ndim > 4) throw invalid("grid dimensionality must be 1..4, got %d", ndim);
    if (n < 1 || !data || !out) throw invalid("data, n >= 1 and out are required");
    PKDE_CUDA_TRY(cudaSetDevice(ctx->device));
    settle_pending(ctx);
    cudaStream_t st = (cudaStream_t)stream;
    DrainOnError drain{ctx, st};
    const double *d_data = data;
    if (!(flags & PKDE_DEVICE_INPUT)) {
      double *dd = (double *)ensure(ctx, BUF_DATA, sizeof(double) * ndim * n);
      copy_in(dd, data, sizeof(double) * ndim * n, false, st);
      d_data = dd;
    }
    const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((n + kThreads - 1) / kThreads, 4 * ctx->sm_count));
    double *m = (double *)ensure(ctx, BUF_MISC, sizeof(double) * (8 + 8 * (size_t)nb));
    {
      ::pkde::Trace _tr(ctx, PKDE_PHASE_OTHER, st);
      extrema_partial_kernel<<<nb, kThreads, 0, st>>>(d_data, n, ndim, m + 8);
    }
    PKDE_CHECK_LAUNCH();
    {
      ::pkde::Trace _tr(ctx, PKDE_PHASE_OTHER, st);
      extrema_final_kernel<<<1, 32, 0, st>>>(m + 8, nb, ndim, m);
    }
    PKDE_CHECK_LAUNCH();
    double ext[8];
    PKDE_CUDA_TRY(cudaMemcpyAsync(ext, m, sizeof(ext), cudaMemcpyDeviceToHost, st));
    PKDE_CUDA_TRY(cudaStreamSynchronize(st));
    pkde_grid g;
    std::memset(&g, 0, sizeof(g));
    g.ndim = ndim;
    for (int j = 0; j < ndim; ++j) {
      const double a = ext[j], b = ext[4 + j];
      if (!std::isfinite(a) || !std::isfinite(b)) throw invalid("samples must be finite");
      const double pad = padding ? padding[j] : 0.1 * std::fabs(b - a);
      const double lo = a - pad, hi0 = b + pad;
      int64_t nj;
      double hi;
      if (steps && !dims) {
        if (!(steps[j] > 0)) throw invalid("grid steps must be positive");
        nj = (int64_t)std::floor((hi0 - lo) / steps[j]) + 1;
        hi = lo + (double)(nj - 1) * steps[j];
      } else {
        nj = dims ? dims[j] : 150;
        hi = hi0;
      }
      if (nj < 2) throw invalid("grid axis %d needs at least 2 points", j + 1);
      g.dims[j] = nj;
      g.lo[j] = lo;
      g.hi[j] = hi;
      g.h[j] = range_step(lo, hi, nj);
    }
    grid_validate(&g);
    *out = g;
  });
}

int pkde_normalize_density(pkde_ctx *ctx, double *density, int64_t G, double dx, uint32_t flags, void *stream) {
  return pkde_guard(ctx, [&] {
    using namespace pkde;
    if (!ctx) throw invalid("context is NULL");
    if (G < 1 || !density) throw invalid("density and G >= 1 are required");
    if (!(dx > 0) || !std::isfinite(dx)) throw invalid("Normalization requires a grid or dx to be specified.");
    PKDE_CUDA_TRY(cudaSetDevice(ctx->device));
    settle_pending(ctx);
    cudaStream_t st = (cudaStream_t)stream;
    DrainOnError drain{ctx, st};
    const bool dev = flags & PKDE_DEVICE_INPUT;
    double *d = density;
    if (!dev) {
      d = (double *)ensure(ctx, BUF_OUT, sizeof(double) * G);
      copy_in(d, density, sizeof(double) * G, false, st);
    }
    const int nb = (int)std::max<int64_t>(1, std::min<int64_t>((G + kThreads - 1) / kThreads, 4 * ctx->sm_count));
    double *partial = (double *)ensure(ctx, BUF_MISC, sizeof(double) * nb);
    {
      ::pkde::Trace _tr(ctx, PKDE_PHASE_OTHER, st);
      sum_partial_kernel<<<nb, kThreads, 0, st>>>(d, G, partial);
    }
    PKDE_CHECK_LAUNCH();
    {
      ::pkde::Trace _tr(ctx, PKDE_PHASE_OTHER, st);
      normalize_kernel<<<nb, kThreads, 0, st>>>(d, G, partial, nb, dx);
    }
    PKDE_CHECK_LAUNCH();
    if (!dev) copy_out(density, d, sizeof(double) * G, false, st);
    PKDE_CUDA_TRY(cudaStreamSynchronize(st));
  });
}

}  // extern "C"
