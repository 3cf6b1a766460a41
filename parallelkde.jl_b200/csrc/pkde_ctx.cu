// Context lifetime, device buffers, argument checks and small C-ABI entry points.
#include <algorithm>
#include <cstring>
#include <limits>
#include <map>
#include <memory>

#include "pkde_internal.cuh"

namespace pkde {

int grid_validate(const pkde_grid *g) {
  if (!g) throw invalid("grid is NULL");
  if (g->ndim < 1 || g->ndim > 4) throw invalid("grid dimensionality must be 1..4, got %d", g->ndim);
  for (int j = 0; j < g->ndim; ++j) {
    if (g->dims[j] < 2) throw invalid("grid axis %d needs at least 2 points", j + 1);
    if (!(g->h[j] > 0.0) || !std::isfinite(g->h[j])) throw invalid("grid spacing of axis %d must be positive", j + 1);
    if (!(g->hi[j] > g->lo[j])) throw invalid("grid bounds of axis %d are empty", j + 1);
    if (g->dims[j] > (1 << 20)) throw invalid("grid axis %d is longer than 2^20 points", j + 1);
  }
  int64_t G = grid_size(g);
  if (G > (int64_t(1) << 31)) throw invalid("grid has more than 2^31 points");
  return 0;
}

int64_t grid_size(const pkde_grid *g) {
  int64_t G = 1;
  for (int j = 0; j < g->ndim; ++j) G *= g->dims[j];
  return G;
}

void *ensure(pkde_ctx *ctx, BufId id, size_t bytes) {
  ctx->buf[id].ensure(bytes ? bytes : 16);
  return ctx->buf[id].ptr;
}

void copy_in(void *dst, const void *src, size_t bytes, bool src_on_device, cudaStream_t st) {
  if (!bytes) return;
  PKDE_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, src_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
}

void copy_out(void *dst, const void *src, size_t bytes, bool dst_on_device, cudaStream_t st) {
  if (!bytes) return;
  PKDE_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, dst_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
}

__global__ void divide_kernel(const double *num, const double *den, double *out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = div_nr(num[i], den[i]);
}

}  // namespace pkde

extern "C" {

int pkde_create(pkde_ctx **out, int device) {
  if (!out) return PKDE_EINVAL;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return PKDE_ECUDA;
  if (device < 0 || device >= ndev) return PKDE_EINVAL;
  if (cudaSetDevice(device) != cudaSuccess) return PKDE_ECUDA;
  pkde_ctx *ctx = new pkde_ctx();
  ctx->device = device;
  cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  ctx->smem_optin = (size_t)optin;
  *out = ctx;
  return PKDE_OK;
}

int pkde_destroy(pkde_ctx *ctx) {
  if (!ctx) return PKDE_OK;
  cudaSetDevice(ctx->device);
  pkde::stop_server(ctx);  // finishes the queued requests first
  cudaDeviceSynchronize();
  for (auto &b : ctx->buf) b.release();
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  if (ctx->engine_flags) cudaFreeHost(ctx->engine_flags);
  delete ctx;
  return PKDE_OK;
}

const char *pkde_last_error(const pkde_ctx *ctx) {
  // NULL: the calling thread's last message of a call made without a context
  const std::string &m = pkde::thread_error(ctx);
  return (ctx || !m.empty()) ? m.c_str() : "no context";
}

int pkde_set_wait_limit(pkde_ctx *ctx, int64_t polls) {
  if (!ctx) return PKDE_EINVAL;
  if (polls < 0) {
    pkde::thread_error(ctx) = "the wait limit must be >= 0 polls";
    return PKDE_EINVAL;
  }
  ctx->wait_limit = polls;
  return PKDE_OK;
}

int pkde_set_fault(pkde_ctx *ctx, int32_t point) {
  if (!ctx) return PKDE_EINVAL;
  if (point != PKDE_FAULT_NONE && point != PKDE_FAULT_AFTER_BINNING) {
    pkde::thread_error(ctx) = "unknown fault point";
    return PKDE_EINVAL;
  }
  ctx->fault_point = point;
  return PKDE_OK;
}

int pkde_diag_divide(pkde_ctx *ctx, const double *num, const double *den, double *out, int64_t n, uint32_t flags,
                     void *stream) {
  return pkde_guard(ctx, [&] {
    using namespace pkde;
    if (!ctx) throw invalid("context is NULL");
    if (n < 0 || (n > 0 && (!num || !den || !out))) throw invalid("num, den and out are required");
    PKDE_CUDA_TRY(cudaSetDevice(ctx->device));
    settle_pending(ctx);
    cudaStream_t st = (cudaStream_t)stream;
    DrainOnError drain{ctx, st};
    if (n == 0) return;
    const bool dev = flags & PKDE_DEVICE_INPUT;
    const size_t bytes = sizeof(double) * (size_t)n;
    const double *dn = num, *dd = den;
    double *dq = out;
    if (!dev) {
      double *b = (double *)ensure(ctx, BUF_MISC, 3 * bytes);
      copy_in(b, num, bytes, false, st);
      copy_in(b + n, den, bytes, false, st);
      dn = b;
      dd = b + n;
      dq = b + 2 * n;
    }
    const unsigned blocks = (unsigned)std::min<int64_t>((n + 255) / 256, (int64_t)ctx->sm_count * 8);
    divide_kernel<<<blocks, 256, 0, st>>>(dn, dd, dq, n);
    PKDE_CHECK_LAUNCH();
    if (!dev) copy_out(out, dq, bytes, false, st);
    PKDE_CUDA_TRY(cudaStreamSynchronize(st));
  });
}

const char *pkde_version(void) { return "pkde_b200 0.1 (sm_100a, FP64 gradepro)"; }

int pkde_gradepro_default_params(pkde_gradepro_params *p, int32_t ndim) {
  if (!p || ndim < 1 || ndim > 4) return PKDE_EINVAL;
  std::memset(p, 0, sizeof(*p));
  const double nan = std::numeric_limits<double>::quiet_NaN();
  p->grid.ndim = ndim;
  p->n_bootstraps = 100;
  p->n_steps = 0;
  p->bw_step = nan;
  for (int j = 0; j < 4; ++j) p->bw_final[j] = nan;
  p->alpha_s = nan;
  p->alpha_os = nan;
  p->eps = nan;
  return PKDE_OK;
}

int64_t pkde_boot_index(uint64_t seed, int64_t n, int64_t b, int64_t j) {
  if (n < 1 || n >= (int64_t(1) << 32)) return -1;
  return pkde::boot_draw(seed, n, b, j);
}

}  // extern "C"
