// FP64 mixed-radix FFT along one grid axis of a batch of complex arrays.
//
// Replaces the cuFFT/FFTW plans of the reference (fourier_statistics!,
// FourierSpace.jl:25-104; ifourier_statistics!, :445-524; plans at
// GradeProEstimator.jl:91, 143, 252, 279-280).  Each CTA stages a tile of lines in
// shared memory (coalesced along grid axis 1), runs Stockham autosort stages of radix
// 8/4/2/3/5 (generic radix for other primes) and writes the tile back.  An optional
// per-element real factor (the separable Gaussian propagator of one axis) is applied
// on load, so propagation costs no extra pass over memory.
#include <algorithm>

#include "pkde_internal.cuh"

namespace pkde {
namespace {

constexpr int kFftThreads = 256;

template <int DIR>
__global__ void __launch_bounds__(kFftThreads) fft_axis_kernel(const double2 *in, double2 *out,
                                                                LineSet ls, FftPlan plan, const double2 *__restrict__ tw,
                                                                const double *__restrict__ f0,
                                                                const double *__restrict__ f1, double s0, double s1,
                                                                int nfac, int tl, int pitch) {
  extern __shared__ double2 smem[];
  double2 *bufA = smem;
  double2 *bufB = smem + (size_t)tl * pitch;
  const int n = ls.n;
  const int64_t nlines = ls.nlines();
  const int64_t L0 = (int64_t)blockIdx.x * tl;
  const int nl = (int)min((int64_t)tl, nlines - L0);
  const bool contiguous = ls.inner == 1;
  const int64_t per_array = ls.inner * ls.outer;

  for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
    int l, k;
    if (contiguous) {
      l = e / n;
      k = e - l * n;
    } else {
      k = e / nl;
      l = e - k * nl;
    }
    const int64_t L = L0 + l;
    double2 v = in[ls.base(L) + (int64_t)k * ls.inner];
    if (nfac) {
      const int64_t a = L / per_array;
      const bool second = nfac == 2 && (a & 1);
      const double *f = second ? f1 : f0;
      const double sc = (second ? s1 : s0) * (f ? f[k] : 1.0);
      v = cscale(v, sc);
    }
    bufA[l * pitch + k] = v;
  }
  __syncthreads();
  double2 *res = smem_fft<DIR>(bufA, bufB, pitch, nl, plan, tw);
  for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
    int l, k;
    if (contiguous) {
      l = e / n;
      k = e - l * n;
    } else {
      k = e / nl;
      l = e - k * nl;
    }
    const int64_t L = L0 + l;
    out[ls.base(L) + (int64_t)k * ls.inner] = res[l * pitch + k];
  }
}

}  // namespace

const double2 *twiddles_device(pkde_ctx *ctx, int n) {
  auto it = ctx->twiddles.find(n);
  if (it != ctx->twiddles.end()) return it->second.as<double2>();
  std::vector<double2> tw = make_twiddles(n);
  DevBuf &b = ctx->twiddles[n];
  b.ensure(sizeof(double2) * n);
  PKDE_CUDA_TRY(cudaMemcpy(b.ptr, tw.data(), sizeof(double2) * n, cudaMemcpyHostToDevice));
  return b.as<double2>();
}

// Lines per CTA: enough to fill ~2048 elements, capped by the shared-memory budget.
int lines_per_cta(int n, int64_t nlines) {
  int tl = std::max(1, 2048 / n);
  if (tl > 16) tl = 16;
  if (tl > nlines) tl = (int)nlines;
  return std::max(tl, 1);
}

size_t fft_smem_bytes(int tl, int pitch) { return sizeof(double2) * 2 * (size_t)tl * pitch; }

void fft_axis(pkde_ctx *ctx, const LineSet &ls, const double2 *in, double2 *out, int dir,
              const double *const *factors, const double *scal, int nfac, cudaStream_t st, int phase) {
  const int n = ls.n;
  const int64_t nlines = ls.nlines();
  if (nlines == 0) return;
  const int tl = lines_per_cta(n, nlines);
  const int pitch = n + 1;
  const size_t smem = fft_smem_bytes(tl, pitch);
  if (smem > ctx->smem_optin)
    throw Error{PKDE_EUNSUPPORTED, "grid axis too long for the shared-memory FFT"};
  FftPlan plan = make_plan(n);
  const double2 *tw = twiddles_device(ctx, n);
  const int64_t blocks = (nlines + tl - 1) / tl;
  if (blocks > 0x7fffffff) throw Error{PKDE_EUNSUPPORTED, "too many FFT lines"};
  const double *f0 = factors ? factors[0] : nullptr;
  const double *f1 = (factors && nfac > 1) ? factors[1] : nullptr;
  const double s0 = scal ? scal[0] : 1.0;
  const double s1 = (scal && nfac > 1) ? scal[1] : s0;
  if (dir < 0) {
    allow_dynamic_smem(ctx, fft_axis_kernel<-1>, smem);
    {
      ::pkde::Trace _tr(ctx, phase, st);
      fft_axis_kernel<-1><<<(unsigned)blocks, kFftThreads, smem, st>>>(in, out, ls, plan, tw, f0, f1, s0, s1, nfac, tl, pitch);
    }
  } else {
    allow_dynamic_smem(ctx, fft_axis_kernel<1>, smem);
    {
      ::pkde::Trace _tr(ctx, phase, st);
      fft_axis_kernel<1><<<(unsigned)blocks, kFftThreads, smem, st>>>(in, out, ls, plan, tw, f0, f1, s0, s1, nfac, tl, pitch);
    }
  }
  PKDE_CHECK_LAUNCH();
}

void fft_nd(pkde_ctx *ctx, int ndim, const int64_t *dims, double2 *data, int64_t batch, int dir, cudaStream_t st,
            int phase) {
  int64_t G = 1;
  for (int j = 0; j < ndim; ++j) G *= dims[j];
  for (int a = 0; a < ndim; ++a) {
    LineSet ls = axis_lines(ndim, dims, a, batch);
    double scal[1] = {1.0 / (double)G};
    const bool scale_here = dir > 0 && a == 0;
    fft_axis(ctx, ls, data, data, dir, nullptr, scale_here ? scal : nullptr, scale_here ? 1 : 0, st, phase);
  }
}

}  // namespace pkde

extern "C" int pkde_fft(pkde_ctx *ctx, int32_t ndim, const int64_t *dims, double *data, int32_t batch,
                        int32_t direction, uint32_t flags, void *stream) {
  return pkde_guard(ctx, [&] {
    using namespace pkde;
    if (!ctx) throw invalid("context is NULL");
    if (ndim < 1 || ndim > 4 || !dims || !data || batch < 1) throw invalid("invalid FFT arguments");
    if (direction != -1 && direction != 1) throw invalid("direction must be -1 or +1");
    PKDE_CUDA_TRY(cudaSetDevice(ctx->device));
    settle_pending(ctx);
    cudaStream_t st = (cudaStream_t)stream;
    DrainOnError drain{ctx, st};
    int64_t G = 1;
    for (int j = 0; j < ndim; ++j) {
      if (dims[j] < 1) throw invalid("invalid FFT size");
      G *= dims[j];
    }
    const size_t bytes = sizeof(double2) * G * batch;
    double2 *d = reinterpret_cast<double2 *>(data);
    const bool on_device = flags & PKDE_DEVICE_INPUT;
    if (!on_device) {
      d = (double2 *)ensure(ctx, BUF_SCRATCH, bytes);
      copy_in(d, data, bytes, false, st);
    }
    fft_nd(ctx, ndim, dims, d, batch, direction, st, PKDE_PHASE_FORWARD_FFT);
    if (!on_device) copy_out(data, d, bytes, false, st);
    PKDE_CUDA_TRY(cudaStreamSynchronize(st));
    collect_trace(ctx);
  });
}
