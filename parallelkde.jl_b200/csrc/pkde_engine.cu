// Persistent dataflow engine for the per-bandwidth-step work of an N-D (N >= 2)
// estimation on power-of-two axes of 16..2048 points.
//
// Work: for every step s the inverse FFT of all bootstrap pairs (z, w arrays) and of the
// full-sample means, then VMR + Welford over bootstraps, then the convergence update.
// It is cut into batches b = (step s, group j): groups 0..J-1 hold g bootstrap pairs
// each, group J is the means.  Each batch runs P = N passes: axis passes over grid axes
// N..2 (pass p works on axis N-1-p), then the final axis-1 pass.  A pass is a set of
// tiles, one tile = one CTA-sized work item.
//
// Schedule: round r holds pass p of batch r - p*D for every p (final passes first), so the
// passes of consecutive batches overlap and every dependency points to an earlier
// round.  CTAs are persistent and take items in this global order from an atomic
// counter; an item waits (bounded spin) only for items taken before it, so progress is
// guaranteed whatever the grid size.
//
// Dependencies: pass p > 0 of batch b needs all tiles of pass p-1 of b; pass 0 of b
// needs the ring slot of batch b - Q released (all final tiles of b - Q done); the
// final tile t of a pair group j > 0 needs tile t of group j - 1 of the same step
// (Welford order over bootstraps); group 0 of step s needs tile t of step s-2's means
// (its state slot); the means tile t of step s needs the means tile t of step s-1
// (convergence order).
//
// Memory: intermediates live in Q ring slots sized to stay in L2; data written by one
// CTA and read by another is loaded with ld.global.cg (L2), never through L1.
#include <cuda/atomic>

#include "pkde_regfft.cuh"
#include "pkde_step.cuh"

namespace pkde {

namespace {

constexpr int kEngineThreads = 256;
constexpr long long kSpinLimit = 20000000;  // ~1-2 s of polling, then the run aborts

struct EngineEst {
  int ndim;
  int logn[4];
  int64_t dims[4];
  int64_t G;
  int npairs, nboot, S, J, g, Q, P;
  const double2 *spectra;
  double2 *slots;
  int64_t slot_elems;
  double *wstate;  // 2 state slots x (mean G, m2 G)
  const double *fz, *fw;
  int64_t tab_stride;
  int64_t aoff[4];
  const double *cw, *vscale, *dlogt;
  double invG, inv_n, eps;
  int64_t steps_low, steps_over;
  StepState cs;
  int64_t NB;            // batches
  int64_t nrounds;
  const int64_t *round_start;  // nrounds + 1 prefix sums of items per round
  int *cnt;              // NB x P completed tiles per (batch, pass)
  int *fin;              // NB x Tf per-tile final-pass done flags
  int Tf;                // final-pass tiles per batch
  int tpi[4];            // axis passes: tiles per work item, by axis
  int D;                 // pass p of batch b runs in round b + p*D
  int *next;             // work counter
  int *error;            // 1: dependency wait timed out
  const double2 *tw[13]; // per-stage twiddle tables by log2(line length)
};

__device__ __forceinline__ int ld_acquire(const int *p) {
  cuda::atomic_ref<int, cuda::thread_scope_device> a(*const_cast<int *>(p));
  return a.load(cuda::memory_order_acquire);
}
__device__ __forceinline__ void add_release(int *p, int v) {
  cuda::atomic_ref<int, cuda::thread_scope_device> a(*p);
  a.fetch_add(v, cuda::memory_order_release);
}

// Spin until *p >= target (thread 0 only).  Returns false on timeout or abort.
__device__ bool wait_geq(const EngineEst &E, const int *p, int target) {
  long long it = 0;
  while (ld_acquire(p) < target) {
    if (++it > kSpinLimit || ld_acquire(E.error)) {
      atomicExch(E.error, 1);
      return false;
    }
    __nanosleep(64);
  }
  return true;
}

__host__ __device__ __forceinline__ int tile_lines_of(int logn) { return (1 << logn) / 8 > 256 ? 1 : 256 * 8 / (1 << logn); }

__host__ __device__ __forceinline__ int batch_arrays(const EngineEst &E, int64_t b) {
  const int j = (int)(b % (E.J + 1));
  if (j == E.J) return 1;
  const int np = min(E.g, E.npairs - j * E.g);
  return 2 * np;
}

__host__ __device__ __forceinline__ int pass_tiles(const EngineEst &E, int64_t b, int p) {
  if (p == E.P - 1) return E.Tf;
  const int a = E.ndim - 1 - p;
  return (int)(batch_arrays(E, b) * (E.G / E.dims[a]) / ((int64_t)tile_lines_of(E.logn[a]) * E.tpi[a]));
}

// ------------------------------------------------------------------ tile bodies
template <int LOGN>
__device__ __forceinline__ void stage_tw(double2 *sm_tw, const double2 *tw_g, int &cached, int key) {
  if (cached != key) {  // uniform across the block
    __syncthreads();
    for (int i = threadIdx.x; i < Pow2<LOGN>::TWSIZE; i += blockDim.x) sm_tw[i] = tw_g[i];
    cached = key;
    __syncthreads();
  }
}

// Inverse FFT of `ntiles` consecutive tiles of NL adjacent lines along an axis >= 2,
// the axis factor applied on load.  Consecutive lanes take adjacent lines (column
// mapping), so every global access moves NL*16 contiguous bytes.  FROM_SPECTRA: the
// input is the read-only spectra, streamed with the evict-first hint so that it does
// not push the ring slots out of L2; otherwise the input is a ring slot written by
// other CTAs and is read through L2 only.
template <int LOGN, bool FROM_SPECTRA>
__device__ void axis_tiles(double2 *smem, const double2 *sm_tw, const double2 *in, double2 *out, int64_t inner,
                           int64_t first_tile, int ntiles, const double *f) {
  using P = Pow2<LOGN>;
  using I = TileIdx<LOGN, true>;
  const int t = I::bfly();
  auto base_of = [&](int u) {
    const int64_t Lw = (first_tile + u) * P::NL + I::line();
    return (Lw / inner) * P::N * inner + (Lw % inner);
  };
  auto load = [&](int64_t base, double2 *x) {
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int64_t off = base + (int64_t)in_pos<LOGN>(t, r) * inner;
      x[r] = FROM_SPECTRA ? __ldcs(in + off) : __ldcg(in + off);
    }
  };
  // the next tile's loads are issued before this tile's FFT, hiding their latency
  double2 nxt[8];
  int64_t base = base_of(0);
  load(base, nxt);
  for (int u = 0; u < ntiles; ++u) {
    double2 v[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) v[r] = cscale(nxt[r], f[in_pos<LOGN>(t, r)]);
    const int64_t nbase = u + 1 < ntiles ? base_of(u + 1) : base;
    if (u + 1 < ntiles) load(nbase, nxt);
    tile_fft_reg<LOGN, 1, true>(smem, v, sm_tw);
#pragma unroll
    for (int i = 0; i < 8; ++i) __stcg(out + base + (int64_t)out_pos<LOGN>(t, i) * inner, v[i]);
    base = nbase;
  }
}

__device__ __forceinline__ double div_nr(double v, double m) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(m));
  double e = fma(-m, y, 1.0);
  y = fma(y, e, y);
  e = fma(-m, y, 1.0);
  y = fma(y, e, y);
  double q = v * y;
  const double rem = fma(-m, q, v);
  return fma(rem, y, q);
}
__device__ __forceinline__ double vmr_of(double Mv, double Vv, double inv_n) {
  const double m = fabs(Mv) * inv_n;
  const double v = fabs(Vv) * inv_n - m * m;
  return div_nr(v, m);
}
__device__ __forceinline__ void welford(double x, double inv, double &mean, double &m2) {
  const double delta = x - mean;
  mean = fma(delta, inv, mean);
  m2 = fma(delta, x - mean, m2);
}

template <int LOGN>
__device__ void vmr_tile(double2 *smem, double2 *state, double2 *sm_tw, const double2 *in, int npairs, int b0,
                         int nboot, const double *fz, const double *fw, double cz, double cw, double inv_n, int64_t G,
                         double *wst, int first, int64_t tile) {
  using P = Pow2<LOGN>;
  using I = TileIdx<LOGN, false>;
  const int64_t rbase = (tile * P::NL + I::line()) * P::N;
  const int t = I::bfly();
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int64_t gi = rbase + out_pos<LOGN>(t, i);
    state[i * kEngineThreads + threadIdx.x] =
        first ? make_double2(0.0, 0.0) : make_double2(__ldcg(wst + gi), __ldcg(wst + G + gi));
  }
  for (int p = 0; p < npairs; ++p) {
    const double2 *zs = in + (int64_t)(2 * p) * G + rbase;
    const double2 *ws = zs + G;
    double2 z[8], w[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int k = in_pos<LOGN>(t, r);
      z[r] = cscale(__ldcg(zs + k), cz * fz[k]);
    }
    tile_fft_reg<LOGN, 1, false>(smem, z, sm_tw);
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int k = in_pos<LOGN>(t, r);
      w[r] = cscale(__ldcg(ws + k), cw * fw[k]);
    }
    tile_fft_reg<LOGN, 1, false>(smem, w, sm_tw);
    const int b = b0 + 2 * p;
    const double inv_a = 1.0 / (double)(b + 1), inv_b = 1.0 / (double)(b + 2);
    const bool has_b = b + 1 < nboot;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      double2 s = state[i * kEngineThreads + threadIdx.x];
      welford(vmr_of(z[i].x, w[i].x, inv_n), inv_a, s.x, s.y);
      if (has_b) welford(vmr_of(z[i].y, w[i].y, inv_n), inv_b, s.x, s.y);
      state[i * kEngineThreads + threadIdx.x] = s;
    }
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int64_t gi = rbase + out_pos<LOGN>(t, i);
    const double2 s = state[i * kEngineThreads + threadIdx.x];
    __stcg(wst + gi, s.x);
    __stcg(wst + G + gi, s.y);
  }
}

template <int LOGN>
__device__ void means_tile(double2 *smem, double2 *sm_tw, const double2 *in, const double *fz, double cz,
                           const double *wst, int64_t G, int nboot, double vscale, double dlogt, double eps,
                           int64_t steps_low, int64_t steps_over, const StepState &cs, int step, int64_t tile) {
  using P = Pow2<LOGN>;
  using I = TileIdx<LOGN, false>;
  const int64_t rbase = (tile * P::NL + I::line()) * P::N;
  const int t = I::bfly();
  double2 z[8];
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int k = in_pos<LOGN>(t, r);
    z[r] = cscale(__ldcg(in + rbase + k), cz * fz[k]);
  }
  tile_fft_reg<LOGN, 1, false>(smem, z, sm_tw);
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int64_t gi = rbase + out_pos<LOGN>(t, i);
    const double mu = sqrt(z[i].x * z[i].x + z[i].y * z[i].y);
    const double m2 = __ldcg(wst + G + gi);
    step_update<true>(cs, gi, mu, vscale * m2 / (double)(nboot - 1), dlogt, eps, steps_low, steps_over, step);
  }
}

// ------------------------------------------------------------------ the engine
struct Decoded {
  int64_t b;
  int p;
  int64_t tile;
};

__device__ bool decode(const EngineEst &E, int64_t item, int64_t &round, Decoded &d) {
  while (round < E.nrounds && E.round_start[round + 1] <= item) ++round;
  if (round >= E.nrounds) return false;
  int64_t off = item - E.round_start[round];
  for (int p = E.P - 1; p >= 0; --p) {
    const int64_t b = round - (int64_t)p * E.D;
    if (b < 0 || b >= E.NB) continue;
    const int n = pass_tiles(E, b, p);
    if (off < n) {
      d.b = b;
      d.p = p;
      d.tile = off;
      return true;
    }
    off -= n;
  }
  return false;
}

#define PKDE_ENGINE_SWITCH(LN, CALL) \
  switch (LN) {                      \
    case 4: CALL(4); break;          \
    case 5: CALL(5); break;          \
    case 6: CALL(6); break;          \
    case 7: CALL(7); break;          \
    case 8: CALL(8); break;          \
    case 9: CALL(9); break;          \
    case 10: CALL(10); break;        \
    case 11: CALL(11); break;        \
    default: break;                  \
  }

__global__ void __launch_bounds__(kEngineThreads, 2) engine_kernel(EngineEst E, int64_t total_items, int max_tile,
                                                                   int max_tw) {
  extern __shared__ double2 smem[];
  double2 *tile_mem = smem;
  double2 *state = smem + max_tile;
  double2 *sm_tw = state + 8 * kEngineThreads;
  __shared__ int64_t s_next;
  __shared__ int s_ok;
  int cached_tw = -1;
  int64_t round = 0;
  (void)max_tw;
  // The next item is taken while the current one runs (items are taken in increasing
  // order per CTA, so every wait still points to an earlier item).
  if (threadIdx.x == 0) s_next = (int64_t)atomicAdd(E.next, 1);
  __syncthreads();
  int64_t item = s_next;
  for (;;) {
    if (item >= total_items) break;
    __syncthreads();  // everyone has read s_next
    if (threadIdx.x == 0) s_next = ld_acquire(E.error) ? total_items : (int64_t)atomicAdd(E.next, 1);
    Decoded d;
    if (!decode(E, item, round, d)) break;
    const int64_t b = d.b;
    const int p = d.p;
    const int64_t s = b / (E.J + 1);
    const int j = (int)(b % (E.J + 1));
    const bool means = j == E.J;
    const int64_t slot = b % E.Q;
    double2 *slot_base = E.slots + slot * E.slot_elems;
    // ---- dependencies (thread 0 spins; acquire orders the data reads after it)
    if (threadIdx.x == 0) {
      bool ok = true;
      if (p == 0) {
        if (b >= E.Q) ok = wait_geq(E, E.cnt + (b - E.Q) * E.P + (E.P - 1), pass_tiles(E, b - E.Q, E.P - 1));
      } else {
        ok = wait_geq(E, E.cnt + b * E.P + (p - 1), pass_tiles(E, b, p - 1));
      }
      if (ok && p == E.P - 1) {
        if (j > 0) ok = wait_geq(E, E.fin + (b - 1) * E.Tf + d.tile, 1);  // Welford order / all groups done
        if (ok && j == 0 && s >= 2)                                         // state slot free
          ok = wait_geq(E, E.fin + ((s - 2) * (E.J + 1) + E.J) * E.Tf + d.tile, 1);
        if (ok && means && s >= 1)                                          // convergence order
          ok = wait_geq(E, E.fin + ((s - 1) * (E.J + 1) + E.J) * E.Tf + d.tile, 1);
      }
      s_ok = ok;
    }
    __syncthreads();
    if (!s_ok) break;
    // ---- work
    const double *fzs = E.fz + s * E.tab_stride;
    const double *fws = E.fw + s * E.tab_stride;
    if (p < E.P - 1) {
      const int a = E.ndim - 1 - p;
      const int ln = E.logn[a];
      const int64_t lines = E.G / E.dims[a];
      const int tpi = E.tpi[a];
      const int64_t ipa = lines / ((int64_t)tile_lines_of(ln) * tpi);  // items per array
      const int64_t arr = d.tile / ipa;
      const int64_t first_tile = (d.tile % ipa) * tpi;
      int64_t inner = 1;
      for (int q = 0; q < a; ++q) inner *= E.dims[q];
      const double2 *in = p == 0 ? (means ? E.spectra + (int64_t)(2 * E.npairs) * E.G
                                          : E.spectra + (int64_t)(2 * j * E.g) * E.G)
                                 : slot_base;
      in += arr * E.G;
      double2 *out = slot_base + arr * E.G;
      const double *f = (!means && (arr & 1)) ? fws + E.aoff[a] : fzs + E.aoff[a];
#define PKDE_AXIS(L)                                                                      \
  {                                                                                       \
    stage_tw<L>(sm_tw, E.tw[L], cached_tw, L);                                            \
    if (p == 0)                                                                           \
      axis_tiles<L, true>(tile_mem, sm_tw, in, out, inner, first_tile, tpi, f);           \
    else                                                                                  \
      axis_tiles<L, false>(tile_mem, sm_tw, in, out, inner, first_tile, tpi, f);          \
  }
      PKDE_ENGINE_SWITCH(ln, PKDE_AXIS)
#undef PKDE_AXIS
    } else {
      const int ln = E.logn[0];
      if (!means) {
        const int np = batch_arrays(E, b) / 2;
#define PKDE_VMR(L)                                                                                         \
  {                                                                                                         \
    stage_tw<L>(sm_tw, E.tw[L], cached_tw, L);                                                              \
    vmr_tile<L>(tile_mem, state, sm_tw, slot_base, np, 2 * j * E.g, E.nboot, fzs + E.aoff[0],               \
                fws + E.aoff[0], E.invG, E.invG * E.cw[s], E.inv_n, E.G, E.wstate + (s & 1) * 2 * E.G,      \
                j == 0, d.tile);                                                                            \
  }
        PKDE_ENGINE_SWITCH(ln, PKDE_VMR)
#undef PKDE_VMR
      } else {
#define PKDE_MEANS(L)                                                                                        \
  {                                                                                                          \
    stage_tw<L>(sm_tw, E.tw[L], cached_tw, L);                                                               \
    means_tile<L>(tile_mem, sm_tw, slot_base, fzs + E.aoff[0], E.invG, E.wstate + (s & 1) * 2 * E.G, E.G,     \
                  E.nboot, E.vscale[s], E.dlogt[s], E.eps, E.steps_low, E.steps_over, E.cs, (int)s, d.tile); \
  }
        PKDE_ENGINE_SWITCH(ln, PKDE_MEANS)
#undef PKDE_MEANS
      }
    }
    // ---- signal completion
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      if (p == E.P - 1) add_release(E.fin + b * E.Tf + d.tile, 1);
      add_release(E.cnt + b * E.P + p, 1);
    }
    item = s_next;
  }
}

int ilog2_pow2(int64_t n) {
  int l = 0;
  while ((int64_t(1) << l) < n) ++l;
  return (int64_t(1) << l) == n ? l : -1;
}

size_t tile_elems(int logn) {
  switch (logn) {
#define PKDE_T(L) \
  case L: return Pow2<L>::TILE;
    PKDE_T(4) PKDE_T(5) PKDE_T(6) PKDE_T(7) PKDE_T(8) PKDE_T(9) PKDE_T(10) PKDE_T(11)
#undef PKDE_T
    default: return 0;
  }
}
size_t tw_elems(int logn) {
  switch (logn) {
#define PKDE_T(L) \
  case L: return Pow2<L>::TWSIZE;
    PKDE_T(4) PKDE_T(5) PKDE_T(6) PKDE_T(7) PKDE_T(8) PKDE_T(9) PKDE_T(10) PKDE_T(11)
#undef PKDE_T
    default: return 0;
  }
}

}  // namespace

const double2 *stage_twiddles_device(pkde_ctx *ctx, int logn);

// Engine schedule parameters; the environment overrides the defaults (tuning runs).
int engine_env_int(const char *name, int dflt, int lo, int hi) {
  const char *v = getenv(name);
  if (!v || !*v) return dflt;
  const int x = atoi(v);
  return x < lo ? lo : (x > hi ? hi : x);
}

bool engine_ok(const pkde_grid *g) {
  if (g->ndim < 2) return false;
  const int64_t G = grid_size(g);
  int64_t inner = 1;
  for (int j = 0; j < g->ndim; ++j) {
    const int ln = ilog2_pow2(g->dims[j]);
    if (ln < 4 || ln > 11) return false;
    const int nl = tile_lines_of(ln);
    if ((G / g->dims[j]) % nl) return false;
    if (j > 0 && inner % nl) return false;
    inner *= g->dims[j];
  }
  return true;
}

void run_engine(pkde_ctx *ctx, const EngineArgs &A, cudaStream_t st) {
  const pkde_grid *g = A.grid;
  EngineEst E{};
  E.ndim = g->ndim;
  E.G = grid_size(g);
  for (int j = 0; j < g->ndim; ++j) {
    E.dims[j] = g->dims[j];
    E.logn[j] = ilog2_pow2(g->dims[j]);
    E.aoff[j] = A.aoff[j];
  }
  E.npairs = A.npairs;
  E.nboot = A.nboot;
  E.S = A.S;
  E.P = g->ndim;
  // pairs per group: ring slot (2g arrays) within 16 MB, at least one pair
  const int64_t arr_bytes = (int64_t)sizeof(double2) * E.G;
  const int64_t slot_mb = engine_env_int("PKDE_ENGINE_SLOT_MB", 8, 1, 256);
  E.g = (int)std::max<int64_t>(1, std::min<int64_t>(E.npairs, (slot_mb << 20) / (2 * arr_bytes)));
  E.J = (E.npairs + E.g - 1) / E.g;
  // pipeline delay between passes of one batch; ring slots cover the delay
  E.D = engine_env_int("PKDE_ENGINE_DELAY", 2, 1, 8);
  E.Q = (E.P - 1) * E.D + 2;
  E.NB = (int64_t)E.S * (E.J + 1);
  E.Tf = (int)((E.G / E.dims[0]) / tile_lines_of(E.logn[0]));
  for (int a = 0; a < 4; ++a) E.tpi[a] = 1;
  for (int a = 1; a < E.ndim; ++a) {
    const int64_t tiles = (E.G / E.dims[a]) / tile_lines_of(E.logn[a]);
    int want = engine_env_int("PKDE_ENGINE_TPI", 2, 1, 16);
    while (want > 1 && tiles % want) want >>= 1;
    E.tpi[a] = want;
  }
  E.nrounds = E.NB + (int64_t)(E.P - 1) * E.D;
  E.slot_elems = (int64_t)2 * E.g * E.G;
  E.spectra = A.spectra;
  E.fz = A.fz;
  E.fw = A.fw;
  E.tab_stride = A.tab_stride;
  E.invG = 1.0 / (double)E.G;
  E.inv_n = A.inv_n;
  E.eps = A.eps;
  E.steps_low = A.steps_low;
  E.steps_over = A.steps_over;
  E.cs = A.cs;
  for (int l = 0; l < 13; ++l) E.tw[l] = nullptr;
  size_t max_tile = 0, max_tw = 1;
  for (int j = 0; j < g->ndim; ++j) {
    E.tw[E.logn[j]] = stage_twiddles_device(ctx, E.logn[j]);
    max_tile = std::max(max_tile, tile_elems(E.logn[j]));
    max_tw = std::max(max_tw, tw_elems(E.logn[j]));
  }
  // schedule: items per round
  std::vector<int64_t> rs(E.nrounds + 1, 0);
  for (int64_t r = 0; r < E.nrounds; ++r) {
    int64_t n = 0;
    for (int p = 0; p < E.P; ++p) {
      const int64_t b = r - (int64_t)p * E.D;
      if (b >= 0 && b < E.NB) n += pass_tiles(E, b, p);
    }
    rs[r + 1] = rs[r] + n;
  }
  const int64_t total = rs[E.nrounds];
  // device memory: [slots][wstate][per-step scalars][round starts][counters]
  const size_t slot_bytes = sizeof(double2) * (size_t)E.Q * E.slot_elems;
  const size_t wst_bytes = sizeof(double) * 4 * (size_t)E.G;
  const size_t sc_bytes = sizeof(double) * 3 * (size_t)E.S;
  const size_t rs_bytes = sizeof(int64_t) * rs.size();
  const size_t cnt_bytes = sizeof(int) * ((size_t)E.NB * E.P + (size_t)E.NB * E.Tf + 2);
  char *m = (char *)ensure(ctx, BUF_SCRATCH, slot_bytes + wst_bytes + sc_bytes + rs_bytes + cnt_bytes + 256);
  E.slots = (double2 *)m;
  E.wstate = (double *)(m + slot_bytes);
  double *sc = (double *)(m + slot_bytes + wst_bytes);
  int64_t *drs = (int64_t *)(m + slot_bytes + wst_bytes + sc_bytes);
  int *cnt = (int *)(m + slot_bytes + wst_bytes + sc_bytes + rs_bytes);
  E.cw = sc;
  E.vscale = sc + E.S;
  E.dlogt = sc + 2 * E.S;
  E.round_start = drs;
  E.cnt = cnt;
  E.fin = cnt + E.NB * E.P;
  E.next = E.fin + E.NB * E.Tf;
  E.error = E.next + 1;
  PKDE_CUDA_TRY(cudaMemcpyAsync(sc, A.cw, sizeof(double) * E.S, cudaMemcpyHostToDevice, st));
  PKDE_CUDA_TRY(cudaMemcpyAsync(sc + E.S, A.vscale, sizeof(double) * E.S, cudaMemcpyHostToDevice, st));
  PKDE_CUDA_TRY(cudaMemcpyAsync(sc + 2 * E.S, A.dlogt, sizeof(double) * E.S, cudaMemcpyHostToDevice, st));
  PKDE_CUDA_TRY(cudaMemcpyAsync(drs, rs.data(), rs_bytes, cudaMemcpyHostToDevice, st));
  PKDE_CUDA_TRY(cudaMemsetAsync(cnt, 0, cnt_bytes, st));
  const size_t smem = sizeof(double2) * (max_tile + 8 * kEngineThreads + max_tw);
  PKDE_CUDA_TRY(cudaFuncSetAttribute(engine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  PKDE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, engine_kernel, kEngineThreads, smem));
  if (per_sm < 1) throw Error{PKDE_EUNSUPPORTED, "engine kernel does not fit on an SM"};
  const int64_t grid = std::min<int64_t>(total, (int64_t)per_sm * ctx->sm_count);
  {
    Trace tr(ctx, PKDE_PHASE_STEP_VMR, st);
    engine_kernel<<<(unsigned)grid, kEngineThreads, smem, st>>>(E, total, (int)max_tile, (int)max_tw);
  }
  PKDE_CHECK_LAUNCH();
  int err = 0;
  PKDE_CUDA_TRY(cudaMemcpyAsync(&err, E.error, sizeof(int), cudaMemcpyDeviceToHost, st));
  PKDE_CUDA_TRY(cudaStreamSynchronize(st));
  if (err) throw Error{PKDE_ECUDA, "step engine: a dependency wait timed out (run aborted)"};
}

}  // namespace pkde
