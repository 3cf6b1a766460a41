// Internal definitions shared by the pkde_b200 CUDA sources: context, status handling,
// device buffers, FP64 complex helpers and the shared-memory mixed-radix FFT.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <array>
#include <exception>
#include <map>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/pkde_b200.h"

namespace pkde {

// ----------------------------------------------------------------------------- status
struct Error {
  int code;
  std::string msg;
};

#define PKDE_CUDA_TRY(expr)                                                                     \
  do {                                                                                          \
    cudaError_t _e = (expr);                                                                    \
    if (_e != cudaSuccess) {                                                                    \
      throw ::pkde::Error{_e == cudaErrorMemoryAllocation ? PKDE_ENOMEM : PKDE_ECUDA,          \
                          std::string(#expr) + ": " + cudaGetErrorString(_e)};                  \
    }                                                                                           \
  } while (0)

// After a kernel launch: the launch's error, with the launching source line.
#define PKDE_STR2(x) #x
#define PKDE_STR(x) PKDE_STR2(x)
#define PKDE_CHECK_LAUNCH()                                                                                \
  do {                                                                                                     \
    cudaError_t _e = cudaGetLastError();                                                                   \
    if (_e != cudaSuccess)                                                                                 \
      throw ::pkde::Error{PKDE_ECUDA, std::string("kernel launch at " __FILE__ ":" PKDE_STR(__LINE__) ": ") + \
                                          cudaGetErrorString(_e)};                                         \
  } while (0)

inline Error invalid(const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  return Error{PKDE_EINVAL, buf};
}

// ------------------------------------------------------------------------ device buffer
// Grow-only device allocation owned by the context; reused across calls.
struct DevBuf {
  void *ptr = nullptr;
  size_t bytes = 0;
  void ensure(size_t want) {
    if (want <= bytes) return;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    PKDE_CUDA_TRY(cudaMalloc(&ptr, want));
    bytes = want;
  }
  template <class T>
  T *as() const {
    return reinterpret_cast<T *>(ptr);
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
  }
};

enum BufId {
  BUF_DATA = 0,     // samples (device copy)
  BUF_IDX,          // bootstrap indices (device copy)
  BUF_PRE_CELL,     // per-sample lower cell
  BUF_PRE_RH,       // per-sample remainders
  BUF_COUNTS,       // per (bootstrap, cell) draw counts
  BUF_FIX,          // fixed-point accumulators
  BUF_SPECTRA,      // paired spectra
  BUF_SCRATCH,      // per-step intermediate
  BUF_WELFORD,      // per-point Welford state
  BUF_STATE,        // convergence state
  BUF_TABLES,       // twiddles, propagation factors, per-step scalars
  BUF_OUT,          // device copies of outputs
  BUF_MISC,         // reductions
  BUF_ENGINE,       // step engine: descriptors, schedule, ring slots, counters
  BUF_BATCH,        // per-estimation buffers of a batch
  BUF_COUNT_
};

}  // namespace pkde

struct pkde_ctx {
  int device = 0;
  pkde::DevBuf buf[pkde::BUF_COUNT_];
  std::map<int, pkde::DevBuf> twiddles;  // per line length
  int sm_count = 0;
  size_t smem_optin = 0;
  // tracing (pkde_set_profiling / pkde_get_stats)
  int profiling = PKDE_PROFILE_OFF;
  int step_path = 0;  // PKDE_STEPS_AUTO / PKDE_STEPS_PER_STEP_LAUNCH
  // engine schedule per shape (pkde_set_autotune): key -> {slot MB, tiles per item, delay}
  bool autotune = true;
  // the tuner may also try ring slots that hold half or all of an estimation's bootstrap
  // pairs when those exceed 64 MB (off for serving lanes, whose memory admission assumes
  // slots of at most 64 MB or one pair)
  bool tune_wide = true;
  bool tune_loaded = false;
  bool recip_ready = false;  // the step engine's table of 1/i is in this device's constant memory
  std::map<std::string, std::array<int, 3>> tune;
  // polls a step-engine dependency wait makes before it gives up (pkde_set_wait_limit)
  int64_t wait_limit = 20000000;
  // host-side fault injection for tests (pkde_set_fault): one-shot
  int fault_point = PKDE_FAULT_NONE;
  // step-engine error flags, copied back without a synchronisation of their own and
  // checked when the call synchronises (check_engine_flags); page-locked
  int *engine_flags = nullptr;
  int engine_flags_used = 0;
  // binning error flags of the estimations of the call in flight (64 ints each, in the
  // page-locked staging buffer), checked after the call's final synchronisation
  const int *bin_flags = nullptr;
  int bin_flags_count = 0;
  // page-locked staging buffer for asynchronous uploads (grow-only)
  void *pinned = nullptr;
  size_t pinned_bytes = 0;
  // serving (pkde_serve.cu): created on the first pkde_submit
  void *server = nullptr;
  int serve_lanes = 2;
  int64_t serve_lane_bytes = 0;
  uint64_t launches = 0;
  uint64_t phase_launches[PKDE_NPHASES] = {};
  double phase_ms[PKDE_NPHASES] = {};
  struct Pending {
    int phase;
    cudaEvent_t a, b;
  };
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> event_pool;
};

namespace pkde {

// Launch accounting: call trace_begin before and trace_end after each kernel launch.
inline cudaEvent_t pooled_event(pkde_ctx *ctx) {
  if (!ctx->event_pool.empty()) {
    cudaEvent_t e = ctx->event_pool.back();
    ctx->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}
struct Trace {
  pkde_ctx *ctx;
  int phase;
  cudaStream_t st;
  cudaEvent_t a = nullptr;
  Trace(pkde_ctx *c, int p, cudaStream_t s) : ctx(c), phase(p), st(s) {
    ctx->launches++;
    ctx->phase_launches[p]++;
    if (ctx->profiling == PKDE_PROFILE_ALL ||
        (ctx->profiling == PKDE_PROFILE_STEPS && p >= PKDE_PHASE_STEP_FFT && p <= PKDE_PHASE_STEP_MEANS)) {
      a = pooled_event(ctx);
      cudaEventRecord(a, st);
    }
  }
  ~Trace() {
    if (a) {
      cudaEvent_t b = pooled_event(ctx);
      cudaEventRecord(b, st);
      ctx->pending.push_back({phase, a, b});
    }
  }
};
// Dynamic shared memory above 48 KB must be allowed per kernel with cudaFuncSetAttribute,
// which sets a property of the kernel for the whole process, not of one launch.  Serving
// lanes launch from several host threads: if each call set the size its own launch
// needs, one thread could lower the limit between another thread's setting and its
// launch, and that launch would fail.  So the limit only grows (under a lock, per kernel
// and device): it is raised to a launch's need when that need is larger, and never
// lowered, so every launch finds at least what it asked for.  A need beyond what the
// device allows next to the kernel's static shared memory is refused.
template <class K>
inline void allow_dynamic_smem(pkde_ctx *ctx, K kernel, size_t bytes) {
  struct Limit {
    size_t cap, set;
  };
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, Limit> limits;
  const void *fn = reinterpret_cast<const void *>(kernel);
  std::lock_guard<std::mutex> lk(mu);
  auto it = limits.find(std::make_pair(fn, ctx->device));
  if (it == limits.end()) {
    cudaFuncAttributes fa;
    PKDE_CUDA_TRY(cudaFuncGetAttributes(&fa, fn));
    const size_t cap = ctx->smem_optin > fa.sharedSizeBytes ? ctx->smem_optin - fa.sharedSizeBytes : 0;
    it = limits.emplace(std::make_pair(fn, ctx->device), Limit{cap, 0}).first;
  }
  Limit &L = it->second;
  if (bytes > L.cap) throw Error{PKDE_EUNSUPPORTED, "a kernel needs more shared memory than an SM offers"};
  if (bytes > L.set) {
    PKDE_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    L.set = bytes;
  }
}

// Fold finished event pairs into phase_ms (call after the stream synchronised).
inline void collect_trace(pkde_ctx *ctx) {
  for (auto &p : ctx->pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) ctx->phase_ms[p.phase] += ms;
    ctx->event_pool.push_back(p.a);
    ctx->event_pool.push_back(p.b);
  }
  ctx->pending.clear();
}

// ------------------------------------------------------------------------ complex FP64
struct cplx {
  double re, im;
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// a * (sign * i)
__device__ __forceinline__ double2 cmul_si(double2 a, int sign) {
  return sign > 0 ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

// ------------------------------------------------------------------------------ FFT plan
constexpr int kMaxStages = 24;

// Division by a run-time invariant divisor d (1 <= d < 2^13) of x < 2^17 with one
// multiply-high and a shift: q = (umulhi(x, m) + x) >> s, s = ceil(log2 d),
// m = floor(2^32 (2^s - d) / d) + 1 (Granlund & Montgomery, "Division by invariant
// integers using multiplication", PLDI 1994).
struct FastDiv {
  uint32_t m, s;
};
inline FastDiv make_fastdiv(uint32_t d) {
  uint32_t s = 0;
  while ((1u << s) < d) ++s;
  return FastDiv{(uint32_t)(((uint64_t(1) << 32) * ((uint64_t(1) << s) - d)) / d + 1), s};
}
__device__ __forceinline__ uint32_t fdiv(uint32_t x, FastDiv f) { return (__umulhi(x, f.m) + x) >> f.s; }

struct FftPlan {
  int n;
  int nstages;
  int radix[kMaxStages];
  FastDiv div_nb[kMaxStages];  // per stage: n / radix
  FastDiv div_ns[kMaxStages];  // per stage: product of the earlier radices
};

// Factor n into Stockham stages: radix 8, 4, 2 for the power-of-two part, then 3, 5,
// 7 and any remaining prime as a generic stage.
inline FftPlan make_plan(int n) {
  FftPlan p{};
  p.n = n;
  int m = n;
  const int pref[] = {8, 4, 2, 3, 5, 7};
  for (int r : pref) {
    while (m % r == 0) {
      p.radix[p.nstages++] = r;
      m /= r;
    }
  }
  for (int q = 11; m > 1 && q * q <= m; q += 2) {
    while (m % q == 0) {
      p.radix[p.nstages++] = q;
      m /= q;
    }
  }
  if (m > 1) p.radix[p.nstages++] = m;
  int ns = 1;
  for (int st = 0; st < p.nstages; ++st) {
    p.div_nb[st] = make_fastdiv((uint32_t)(n / p.radix[st]));
    p.div_ns[st] = make_fastdiv((uint32_t)ns);
    ns *= p.radix[st];
  }
  return p;
}

// Twiddle table w[m] = (cos(2 pi m / n), sin(2 pi m / n)), m in [0, n), computed in
// long double and rounded once.
inline std::vector<double2> make_twiddles(int n) {
  std::vector<double2> tw(n);
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int m = 0; m < n; ++m) {
    long double a = two_pi * (long double)m / (long double)n;
    tw[m] = make_double2((double)cosl(a), (double)sinl(a));
  }
  return tw;
}

// -------------------------------------------------------------- radix-R butterflies
// DFT of R values in place: X[q] = sum_r v[r] exp(DIR * 2 pi i q r / R).
template <int DIR>
__device__ __forceinline__ void dft2(double2 *v) {
  double2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <int DIR>
__device__ __forceinline__ void dft4(double2 *v) {
  double2 t0 = cadd(v[0], v[2]);
  double2 t1 = csub(v[0], v[2]);
  double2 t2 = cadd(v[1], v[3]);
  double2 t3 = cmul_si(csub(v[1], v[3]), DIR);
  v[0] = cadd(t0, t2);
  v[2] = csub(t0, t2);
  v[1] = cadd(t1, t3);
  v[3] = csub(t1, t3);
}

template <int DIR>
__device__ __forceinline__ void dft8(double2 *v) {
  const double h = 0.70710678118654752440;  // sqrt(1/2)
  double2 e[4] = {v[0], v[2], v[4], v[6]};
  double2 o[4] = {v[1], v[3], v[5], v[7]};
  dft4<DIR>(e);
  dft4<DIR>(o);
  // W8^k, W8 = exp(DIR * 2 pi i / 8)
  double2 o1 = make_double2(h * (o[1].x - DIR * o[1].y), h * (o[1].y + DIR * o[1].x));
  double2 o2 = cmul_si(o[2], DIR);
  double2 o3 = make_double2(h * (-o[3].x - DIR * o[3].y), h * (-o[3].y + DIR * o[3].x));
  v[0] = cadd(e[0], o[0]);
  v[4] = csub(e[0], o[0]);
  v[1] = cadd(e[1], o1);
  v[5] = csub(e[1], o1);
  v[2] = cadd(e[2], o2);
  v[6] = csub(e[2], o2);
  v[3] = cadd(e[3], o3);
  v[7] = csub(e[3], o3);
}

template <int DIR>
__device__ __forceinline__ void dft3(double2 *v) {
  const double s3 = 0.86602540378443864676;  // sin(2 pi / 3)
  double2 t = cadd(v[1], v[2]);
  double2 d = csub(v[1], v[2]);
  double2 m = make_double2(v[0].x - 0.5 * t.x, v[0].y - 0.5 * t.y);
  double2 rot = cmul_si(cscale(d, s3), DIR);
  v[0] = cadd(v[0], t);
  v[1] = cadd(m, rot);
  v[2] = csub(m, rot);
}

template <int DIR>
__device__ __forceinline__ void dft5(double2 *v) {
  const double c1 = 0.30901699437494742410, c2 = -0.80901699437494742410;
  const double s1 = 0.95105651629515357212, s2 = 0.58778525229247312917;
  double2 a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
  double2 a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
  double2 x0 = v[0];
  double2 p1 = make_double2(x0.x + c1 * a1.x + c2 * a2.x, x0.y + c1 * a1.y + c2 * a2.y);
  double2 p2 = make_double2(x0.x + c2 * a1.x + c1 * a2.x, x0.y + c2 * a1.y + c1 * a2.y);
  double2 q1 = cmul_si(make_double2(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y), DIR);
  double2 q2 = cmul_si(make_double2(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y), DIR);
  v[0] = cadd(x0, cadd(a1, a2));
  v[1] = cadd(p1, q1);
  v[4] = csub(p1, q1);
  v[2] = cadd(p2, q2);
  v[3] = csub(p2, q2);
}

__device__ __forceinline__ double2 twiddle(const double2 *tw, int m, int dir) {
  double2 w = tw[m];
  return make_double2(w.x, dir * w.y);
}

// One Stockham stage of radix R over `nlines` lines held in shared memory
// (line pitch `pitch` complex values).  src -> dst.
// Shared-memory layout of the intermediate buffers: within each aligned block of 8
// values the index is XOR-swizzled by the block number (i ^ ((i >> 3) & 7)) when n is a
// multiple of 8.  A first stage (Ns = 1) stores butterfly j's outputs at j*R + q, a
// stride of R*16 bytes that puts every lane of a quarter-warp in one bank group; the
// swizzle spreads them over the 8 groups.  The caller-visible input and output buffers
// keep the plain layout (the first stage reads plain, the last stage writes plain).
__device__ __forceinline__ int swz(int i, bool on) { return on ? (i ^ ((i >> 3) & 7)) : i; }

// Lines of n < 8192 points and at most 16 lines use the plan's multiply-high divisions
// for the butterfly indices (their range limits hold there); longer lines divide.
template <int DIR, int R>
__device__ __forceinline__ void stockham_stage(const double2 *src, double2 *dst, int n, int pitch,
                                               int nlines, int Ns, const double2 *tw, FastDiv dnb, FastDiv dns,
                                               bool swz_src, bool swz_dst) {
  const int nb = n / R;
  const int tstep = n / (Ns * R);
  const bool fast = n < 8192 && nlines <= 16;
  for (int t = threadIdx.x; t < nlines * nb; t += blockDim.x) {
    const int l = fast ? (int)fdiv((uint32_t)t, dnb) : t / nb;
    const int j = t - l * nb;
    const int jq = fast ? (int)fdiv((uint32_t)j, dns) : j / Ns;
    const int k = j - jq * Ns;
    const double2 *s = src + l * pitch;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      double2 x = s[swz(j + r * nb, swz_src)];
      if (r > 0 && k > 0) x = cmul(x, twiddle(tw, r * k * tstep, DIR));
      v[r] = x;
    }
    if constexpr (R == 2) dft2<DIR>(v);
    if constexpr (R == 4) dft4<DIR>(v);
    if constexpr (R == 8) dft8<DIR>(v);
    if constexpr (R == 3) dft3<DIR>(v);
    if constexpr (R == 5) dft5<DIR>(v);
    const int d = jq * Ns * R + k;
    double2 *o = dst + l * pitch;
#pragma unroll
    for (int q = 0; q < R; ++q) o[swz(d + q * Ns, swz_dst)] = v[q];
  }
}

// Generic radix (any R): one thread per output value, O(R) work each.
template <int DIR>
__device__ __forceinline__ void stockham_stage_generic(const double2 *src, double2 *dst, int n,
                                                       int pitch, int nlines, int Ns, int R,
                                                       const double2 *tw, bool swz_src, bool swz_dst) {
  const int nb = n / R;
  const int tstep = n / (Ns * R);
  for (int t = threadIdx.x; t < nlines * n; t += blockDim.x) {
    const int l = t / n;
    const int u = t - l * n;
    const int j = u / R;
    const int q = u - j * R;
    const int k = j % Ns;
    const double2 *s = src + l * pitch;
    const int base = k * tstep + q * nb;  // exponent per input index r
    double2 acc = make_double2(0.0, 0.0);
    int m = 0;
    for (int r = 0; r < R; ++r) {
      double2 x = s[swz(j + r * nb, swz_src)];
      double2 w = twiddle(tw, m, DIR);
      acc.x += x.x * w.x - x.y * w.y;
      acc.y += x.x * w.y + x.y * w.x;
      m += base;
      if (m >= n) m -= n;
    }
    const int d = (j / Ns) * Ns * R + k;
    dst[l * pitch + swz(d + q * Ns, swz_dst)] = acc;
  }
}

// Full FFT of `nlines` lines in shared memory.  Data starts in bufA; returns the
// buffer holding the result (bufA or bufB).  Ends with __syncthreads().
template <int DIR>
__device__ double2 *smem_fft(double2 *bufA, double2 *bufB, int pitch, int nlines, const FftPlan &plan,
                             const double2 *tw) {
  double2 *src = bufA, *dst = bufB;
  int Ns = 1;
  const int n = plan.n;
  const bool sw = (n & 7) == 0;
  for (int st = 0; st < plan.nstages; ++st) {
    const int R = plan.radix[st];
    const bool ss = sw && st > 0, sd = sw && st + 1 < plan.nstages;
    switch (R) {
      case 8: stockham_stage<DIR, 8>(src, dst, n, pitch, nlines, Ns, tw, plan.div_nb[st], plan.div_ns[st], ss, sd); break;
      case 4: stockham_stage<DIR, 4>(src, dst, n, pitch, nlines, Ns, tw, plan.div_nb[st], plan.div_ns[st], ss, sd); break;
      case 2: stockham_stage<DIR, 2>(src, dst, n, pitch, nlines, Ns, tw, plan.div_nb[st], plan.div_ns[st], ss, sd); break;
      case 3: stockham_stage<DIR, 3>(src, dst, n, pitch, nlines, Ns, tw, plan.div_nb[st], plan.div_ns[st], ss, sd); break;
      case 5: stockham_stage<DIR, 5>(src, dst, n, pitch, nlines, Ns, tw, plan.div_nb[st], plan.div_ns[st], ss, sd); break;
      default: stockham_stage_generic<DIR>(src, dst, n, pitch, nlines, Ns, R, tw, ss, sd); break;
    }
    __syncthreads();
    double2 *tmp = src;
    src = dst;
    dst = tmp;
    Ns *= R;
  }
  return src;
}

// Lines along one grid axis of a batch of complex arrays:
// line L -> (array a, outer o, inner i); element k at a*array_stride + (o*n + k)*inner + i.
struct LineSet {
  int n;
  int64_t inner;
  int64_t outer;
  int64_t arrays;
  int64_t array_stride;
  __host__ __device__ int64_t nlines() const { return arrays * outer * inner; }
  __host__ __device__ int64_t base(int64_t L) const {
    int64_t i = L % inner;
    int64_t r = L / inner;
    int64_t o = r % outer;
    int64_t a = r / outer;
    return a * array_stride + o * (int64_t)n * inner + i;
  }
};

inline LineSet axis_lines(int ndim, const int64_t *dims, int axis, int64_t arrays) {
  LineSet ls{};
  ls.n = (int)dims[axis];
  int64_t inner = 1, outer = 1, G = 1;
  for (int j = 0; j < ndim; ++j) G *= dims[j];
  for (int j = 0; j < axis; ++j) inner *= dims[j];
  for (int j = axis + 1; j < ndim; ++j) outer *= dims[j];
  ls.inner = inner;
  ls.outer = outer;
  ls.arrays = arrays;
  ls.array_stride = G;
  return ls;
}

// The bootstrap draw of the counter-based generator (0-based); see pkde_b200.h.
__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ int64_t boot_draw(uint64_t seed, int64_t n, int64_t b, int64_t j) {
  uint64_t x = seed + (uint64_t)(b * n + j + 1) * 0x9E3779B97F4A7C15ull;
  uint64_t z = splitmix64(x);
  return (int64_t)(((z >> 32) * (uint64_t)n) >> 32);
}

// ---------------------------------------------------------------- host-side helpers
int grid_validate(const pkde_grid *g);
int64_t grid_size(const pkde_grid *g);
void *ensure(pkde_ctx *ctx, BufId id, size_t bytes);
void copy_in(void *dst, const void *src, size_t bytes, bool src_on_device, cudaStream_t st);
void copy_out(void *dst, const void *src, size_t bytes, bool dst_on_device, cudaStream_t st);

// FFT driver (pkde_fft.cu): in-place N-D transform of `batch` complex arrays.
// Argument checks of one :gradepro estimation (pkde_gradepro.cu); serving loop teardown
// (pkde_serve.cu).
void validate_gradepro_params(const pkde_gradepro_params *p, int64_t n);
void stop_server(pkde_ctx *ctx);

// Binning of one estimation into the paired spectra layout (pkde_binning.cu), in two
// phases around one host read-back of misc[0..1] (error bits, largest count).
struct DiracJob {
  const pkde_grid *g = nullptr;
  const double *d_data = nullptr;
  int64_t n = 0;
  const int32_t *d_idx = nullptr;
  int64_t nboot = 0;
  uint64_t seed = 0;
  double2 *paired_out = nullptr;
  uint32_t *cell = nullptr;
  double *rh = nullptr;
  uint32_t *counts = nullptr;
  uint32_t *pos = nullptr, *cell_sorted = nullptr;  // samples in lower-cell order
  uint32_t *cstart = nullptr, *cfill = nullptr, *csum = nullptr;
  uint32_t *mult = nullptr;  // nboot x n draws per sample (cell order)
  // low parts of the two-part fixed point: per sample and corner (signed), and the sums
  // (one 64-bit word per real value of the paired spectra)
  long long *qm_lo = nullptr, *qv_lo = nullptr;
  unsigned long long *acc_lo = nullptr;
  int *misc = nullptr;  // 256-byte device block
  int64_t corner_off_h[16] = {};
};
size_t dirac_job_scratch(const pkde_grid *g, int64_t n, int64_t nboot);
void dirac_job_bind(DiracJob &j, char *scratch, int *misc);
void dirac_job_phase_a(pkde_ctx *ctx, DiracJob &j, cudaStream_t st);
// hmisc: misc[0..1] read back (checked here), or nullptr: the caller checks the error flags
// (binning_flags_check) after the call has synchronised; the scales come from the device.
void dirac_job_phase_b(pkde_ctx *ctx, DiracJob &j, const int *hmisc, cudaStream_t st);
void binning_flags_check(const int *hmisc);

void fft_nd(pkde_ctx *ctx, int ndim, const int64_t *dims, double2 *data, int64_t batch, int dir,
            cudaStream_t st, int phase);
// Device twiddle table for size n (cached per context).
const double2 *twiddles_device(pkde_ctx *ctx, int n);
// Launch one axis pass: out[line] = FFT_dir(in[line] * factor), factor per element k of the
// axis taken from factors[a % nfac][k] * scal[a % nfac] (factors may be null).
void fft_axis(pkde_ctx *ctx, const LineSet &ls, const double2 *in, double2 *out, int dir,
              const double *const *factors, const double *scal, int nfac, cudaStream_t st, int phase);

// binning (pkde_binning.cu): fills spectra-ready FP64 arrays
struct BinResult {
  double *means;   // G x nb
  double *sq;      // G x nb (null if not requested)
  uint32_t *counts;
};
void dirac_device(pkde_ctx *ctx, const pkde_grid *g, const double *d_data, int64_t n,
                  const int32_t *d_idx, int64_t nboot, bool identity, uint64_t seed, double *d_means,
                  double *d_sq, uint32_t *d_counts, cudaStream_t st);

}  // namespace pkde

// The calling thread's last error message on a context (pkde_last_error): per thread,
// so that threads sharing a context (pkde_submit / pkde_wait) never race on it.  Entry
// points that accept a NULL context keep their message under the NULL key.
namespace pkde {
inline std::string &thread_error(const pkde_ctx *ctx) {
  thread_local std::unordered_map<const pkde_ctx *, std::string> errs;
  return errs[ctx];
}

// A call that failed after queuing work may leave device work in flight and error-flag
// copies into page-locked memory outstanding (the flags are checked only when a call
// reaches its final synchronisation).  Entry points that reuse the context's buffers
// call this first: with flags outstanding it waits for the device and forgets them.
inline void settle_pending(pkde_ctx *ctx) {
  if (ctx->engine_flags_used || ctx->bin_flags_count) {
    PKDE_CUDA_TRY(cudaDeviceSynchronize());
    ctx->engine_flags_used = 0;
    ctx->bin_flags_count = 0;
  }
}

// Declared by an entry point once its stream is known: if the call leaves by an
// exception, the work it already queued on that stream finishes before the error is
// returned (so no kernel of a failed call still uses the context's buffers when the
// caller goes on), and its outstanding error flags are discarded.
struct DrainOnError {
  pkde_ctx *ctx;
  cudaStream_t st;
  int live = std::uncaught_exceptions();
  ~DrainOnError() {
    if (std::uncaught_exceptions() > live) {
      cudaStreamSynchronize(st);
      if (ctx) {
        ctx->engine_flags_used = 0;
        ctx->bin_flags_count = 0;
      }
    }
  }
};

// Host-side fault injection (pkde_set_fault): throws once at the armed point.
inline void fault_point(pkde_ctx *ctx, int point) {
  if (ctx->fault_point == point) {
    ctx->fault_point = PKDE_FAULT_NONE;
    throw Error{PKDE_ECUDA, "injected host fault (pkde_set_fault)"};
  }
}

// v / m without the IEEE division subroutine: the hardware reciprocal estimate refined
// by one Newton-Raphson iteration y <- y + y (1 - m y) (which squares its relative
// error), the quotient q = v y, then one correction q + (v - m q) y with the exact
// remainder from an FMA (P. Markstein, "Computation of elementary functions on the IBM
// RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990; the same correction step
// as in his IA-64 division).  The correction multiplies the errors of q and y, so one
// iteration suffices for a result within an ulp (measured against IEEE division by the
// tests).  For |m| in [2^-1020, 2^1022) (so that 1/m is normal and
// the estimate is not flushed) and a finite normal quotient the result is within 1 ulp of
// the IEEE quotient (2 ulp is the bound the tests assert).  Elsewhere (m zero, subnormal or huge, v or the result not
// finite) it returns the IEEE quotient v / m itself, so it never differs in kind.
__device__ __forceinline__ double div_nr(double v, double m) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(m));
  const double e = fma(-m, y, 1.0);
  y = fma(y, e, y);
  const double q = v * y;
  const double rem = fma(-m, q, v);
  const double r = fma(rem, y, q);
  // range tests on the biased exponents (integer pipe, not the FP64 one): |m| in
  // [2^-1020, 2^1022) and r finite and normal, else the IEEE quotient
  const unsigned em = ((unsigned)__double2hiint(m) >> 20) & 0x7ffu;
  const unsigned er = ((unsigned)__double2hiint(r) >> 20) & 0x7ffu;
  if (em - 3u > 2041u || er - 1u > 2045u) return __ddiv_rn(v, m);
  return r;
}
}  // namespace pkde

// Entry-point wrapper: converts exceptions into status codes + the thread's last error
// (kept under the NULL key when the call has no context).
template <class F>
static int pkde_guard(pkde_ctx *ctx, F &&f) {
  try {
    f();
    return PKDE_OK;
  } catch (const pkde::Error &e) {
    pkde::thread_error(ctx) = e.msg;
    return e.code;
  } catch (const std::exception &e) {
    pkde::thread_error(ctx) = e.what();
    return PKDE_ECUDA;
  }
}
