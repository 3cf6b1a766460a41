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
// Memory: intermediates live in Q ring slots whose size the autotuner picks per shape
// (8-64 MB, or slots holding half or all of the bootstrap pairs: then the ring exceeds
// the L2 and the intermediates round-trip through HBM); data written by one CTA and
// read by another is loaded with ld.global.cg (L2), never through L1.
#include <cuda/atomic>

#include <algorithm>
#include <array>
#include <cstdio>
#include <cstring>
#include <string>

#include "pkde_regfft.cuh"
#include "pkde_step.cuh"

namespace pkde {

namespace {

#ifndef PKDE_ENGINE_THREADS
#define PKDE_ENGINE_THREADS 256
#endif
// Threads per CTA; CTAs per SM (registers: kEngineThreads x kEngineCtas x 128 = 64K).
constexpr int kEngineThreads = PKDE_ENGINE_THREADS;
constexpr int kEngineCtas = 512 / kEngineThreads;
// Lines per register tile: one butterfly per thread (the longest line of the register
// path, 8 * kEngineThreads points, is one line per tile).
template <int LOGN>
constexpr int kEL = (1 << LOGN) / 8 >= kEngineThreads ? 1 : kEngineThreads * 8 / (1 << LOGN);
template <int LOGN>
using EP = Pow2<LOGN, kEL<LOGN>>;

// One estimation's part of a launch (device-resident descriptor).
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
  int64_t NB;                  // batches
  int64_t nrounds;             // local rounds
  const int64_t *round_start;  // nrounds + 1 prefix sums of items per local round
  int *cnt;                    // NB x P completed tiles per (batch, pass)
  int *fin;                    // NB x Tf per-tile final-pass done flags
  int Tf;                      // final-pass tiles per batch
  int tpi[4];                  // axis passes: tiles per work item, by axis
  int D;                       // pass p of batch b runs in local round b + p*D
  int tl[4];                   // lines per tile, by axis
  int gen[4];                  // 1: the axis uses the shared-memory mixed-radix FFT (any length)
  const double2 *twg[4];       // generic axes: twiddle table (cos, sin)(2 pi m / n), m < n
  const FftPlan *plan;         // generic axes: Stockham radix sequence, by axis (device memory: the
                               // descriptor is copied into shared memory per estimation, and the
                               // plans are ~2 KB that only generic axes read)
  FastDiv dlen[4];             // generic axes: division by the line length
  int mixr[4];                 // mixed-radix axes (gen 2): R of N = R * 2^logn
  const double2 *twc[4];       // mixed-radix axes: combine twiddles W_N^(n1 k2), n1 = 1..R-1
};

// A launch over one or more estimations.  Estimation e runs its local round r in global
// round start_e + r; the global item order is round-major, and within a global round
// estimation-major.  Segment k covers items [seg_start[k], seg_start[k+1]) = the items
// of local round seg[k].y of estimation seg[k].x.  Every dependency of an item is an
// item of the same estimation in an earlier local round, hence earlier in this order.
struct EngineRun {
  const EngineEst *est;
  int count;
  const int64_t *seg_start;  // nseg + 1
  const int2 *seg;           // nseg
  int64_t nseg;
  int64_t total_items;
  int *next;   // work counter
  int *error;  // 1: dependency wait timed out
  long long spin_limit;  // polls per dependency wait (pkde_set_wait_limit), then the run aborts
  const double2 *tw[13];  // per-stage twiddle tables by log2(line length)
};

__device__ __forceinline__ int ld_acquire(const int *p) {
  cuda::atomic_ref<int, cuda::thread_scope_device> a(*const_cast<int *>(p));
  return a.load(cuda::memory_order_acquire);
}
__device__ __forceinline__ void add_release(int *p, int v) {
  cuda::atomic_ref<int, cuda::thread_scope_device> a(*p);
  a.fetch_add(v, cuda::memory_order_release);
}

// Bring `bytes` (a multiple of 16, 16-byte aligned) at p into L2 without waiting for it
// (bulk prefetch; no registers or shared memory involved).
__device__ __forceinline__ void prefetch_l2(const void *p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Final pass over the pairs of a batch: the z and w rows of a tile (contiguous, `tile_elems`
// values from `first`) of pair q are fetched into L2 while pair q - 1 is transformed, so
// that the loads of the next pair hit L2 (measured on 512 x 512 / B = 64: 5 % off the
// engine).  Thread 0 issues it.
__device__ __forceinline__ void prefetch_pair(const double2 *in, int64_t G, int q, int npairs, int64_t first,
                                              int64_t tile_elems) {
  if (threadIdx.x == 0 && q < npairs) {
    prefetch_l2(in + (int64_t)(2 * q) * G + first, (uint32_t)(tile_elems * sizeof(double2)));
    prefetch_l2(in + (int64_t)(2 * q + 1) * G + first, (uint32_t)(tile_elems * sizeof(double2)));
  }
}

// Spin until *p >= target (thread 0 only), at most `limit` polls of about 0.1 us.
// Returns false on timeout (the launch's error flag is set) or when another CTA has
// already aborted the launch.
__device__ bool wait_geq(int *error, const int *p, int target, long long limit) {
  long long it = 0;
  while (ld_acquire(p) < target) {
    if (++it > limit || ld_acquire(error)) {
      atomicExch(error, 1);
      return false;
    }
    __nanosleep(64);
  }
  return true;
}

__host__ __device__ __forceinline__ int tile_lines_of(int logn) {
  return (1 << logn) / 8 >= kEngineThreads ? 1 : kEngineThreads * 8 / (1 << logn);
}

__host__ __device__ __forceinline__ int batch_arrays(const EngineEst &E, int64_t b) {
  const int j = (int)(b % (E.J + 1));
  if (j == E.J) return 1;
  const int np = min(E.g, E.npairs - j * E.g);
  return 2 * np;
}

__host__ __device__ __forceinline__ int pass_tiles(const EngineEst &E, int64_t b, int p) {
  if (p == E.P - 1) return E.Tf;
  const int a = E.ndim - 1 - p;
  return (int)(batch_arrays(E, b) * (E.G / E.dims[a]) / ((int64_t)E.tl[a] * E.tpi[a]));
}

// The propagation factor is separable, P(k) = prod_a f_a(k_a), and every factor but that of
// a line's own axis is constant along the line.  So the first pass of a batch (along the
// last axis, reading the spectra) applies all of them, with the array's scalar (1/G of the
// inverse transform, times the second-moment scale for w arrays); the later passes load
// their inputs as they are.
struct PassScale {
  const double *tab;  // the step's factor tables of the array kind (fz or fw)
  double c;           // 1/G, times cw[s] for the second-moment arrays
};

// c times the factors of every axis but the last at line Lw of a pass-0 line set (Lw:
// linear index over axes 1..N-1, axis 1 fastest).
__device__ __forceinline__ double line_scale(const EngineEst &E, const PassScale &ps, int64_t Lw) {
  double f = ps.c;
  for (int q = 0; q < E.ndim - 1; ++q) {
    int64_t k;
    if (E.gen[q] == 0) {  // power-of-two axis
      k = Lw & (E.dims[q] - 1);
      Lw >>= E.logn[q];
    } else {
      k = Lw % E.dims[q];
      Lw /= E.dims[q];
    }
    f *= ps.tab[E.aoff[q] + k];
  }
  return f;
}

// ------------------------------------------------------------------ tile bodies
template <int LOGN>
__device__ __forceinline__ void stage_tw(double2 *sm_tw, const double2 *tw_g, int &cached, int key) {
  if (cached != key) {  // uniform across the block
    __syncthreads();
    for (int i = threadIdx.x; i < EP<LOGN>::TWSIZE; i += blockDim.x) sm_tw[i] = tw_g[i];
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
__device__ void axis_tiles(double2 *smem, double2 *smem2, const double2 *sm_tw, const double2 *in, double2 *out,
                           int64_t inner, int64_t first_tile, int ntiles, const double *f, const EngineEst &E,
                           const PassScale ps) {
  using P = EP<LOGN>;
  using I = TileIdx<LOGN, true, kEL<LOGN>>;
  const int t = I::bfly();
  // The thread's line Lw = (first_tile + u) NL + line() starts at (Lw / inner) N inner +
  // Lw % inner; quotient and remainder advance by NL lines per tile (no division per tile).
  // Element k of the line is k inner further; its butterfly's elements are t + c (c a
  // compile-time constant of the position), so every offset is tin + c inner.
  const int64_t plane = (int64_t)P::N * inner;
  const int64_t Lw0 = first_tile * P::NL + I::line();
  int64_t lq = Lw0 / inner, lr = Lw0 % inner;
  const int64_t tin = (int64_t)t * inner;
  auto load = [&](int64_t base, double2 *x) {
    const double2 *p = in + base + tin;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const double2 *q = p + (int64_t)(in_pos<LOGN>(t, r) - t) * inner;
      x[r] = FROM_SPECTRA ? __ldcs(q) : __ldcg(q);
    }
  };
  // The next tile's rows are brought into L2 (bulk prefetch, no registers) while this tile
  // is transformed: with its NL lines adjacent in memory (inner a multiple of NL) a tile
  // is N segments of NL * 16 contiguous bytes.  Holding the next tile in registers instead
  // spilled registers to local memory.
  const bool pf = inner % P::NL == 0;
  int64_t base = lq * plane + lr;
  for (int u = 0; u < ntiles; ++u) {
    double2 v[8];
    load(base, v);
    int64_t nbase = base;
    if (u + 1 < ntiles) {
      lr += P::NL;
      while (lr >= inner) lr -= inner, ++lq;
      nbase = lq * plane + lr;
    }
    if (pf && u + 1 < ntiles) {  // the tile's first line starts I::line() elements earlier
      const double2 *b0 = in + nbase - I::line();
      for (int k = threadIdx.x; k < P::N; k += kEngineThreads)
        prefetch_l2(b0 + (int64_t)k * inner, (uint32_t)(P::NL * sizeof(double2)));
    }
    if constexpr (FROM_SPECTRA) {
      const double ncl = line_scale(E, ps, (first_tile + u) * P::NL + I::line());
#pragma unroll
      for (int r = 0; r < 8; ++r) v[r] = cscale(v[r], f[in_pos<LOGN>(t, r)] * ncl);
    }
    tile_fft_reg<LOGN, 1, true, kEL<LOGN>, true>(smem, v, sm_tw, smem2);
    double2 *o = out + base + tin;
#pragma unroll
    for (int i = 0; i < 8; ++i) __stcg(o + (int64_t)(out_pos<LOGN>(t, i) - t) * inner, v[i]);
    base = nbase;
  }
}

// VMR of one bootstrap at one point (DirectSpace.jl:550-552; 1/n as a product, the
// quotient by div_nr).
__device__ __forceinline__ double vmr_of(double Mv, double Vv, double inv_n) {
  const double m = fabs(Mv) * inv_n;
  const double v = fabs(Vv) * inv_n - m * m;
  return div_nr(v, m);
}
// 1/i for the Welford updates over bootstraps i = 1..kRecip-1, each the IEEE quotient
// (filled once per device from the host's division): the final pass reads it with a
// CTA-uniform index instead of dividing twice per pair in every thread.
constexpr int kRecip = 4096;
__constant__ double c_recip[kRecip];
__device__ __forceinline__ double recip_of(int i) { return i < kRecip ? c_recip[i] : 1.0 / (double)i; }

__device__ __forceinline__ void welford(double x, double inv, double &mean, double &m2) {
  const double delta = x - mean;
  mean = fma(delta, inv, mean);
  m2 = fma(delta, x - mean, m2);
}

template <int LOGN>
__device__ void vmr_tile(double2 *smem, double2 *state, double2 *sm_tw, const double2 *in, int npairs, int b0,
                         int nboot, double inv_n, int64_t G, double *wst, int first, int64_t tile) {
  using P = EP<LOGN>;
  using I = TileIdx<LOGN, false, kEL<LOGN>>;
  const int64_t rbase = (tile * P::NL + I::line()) * P::N;
  const int t = I::bfly();
  prefetch_pair(in, G, 0, npairs, tile * P::NL * P::N, P::NL * P::N);
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int64_t gi = rbase + out_pos<LOGN>(t, i);
    state[i * kEngineThreads + threadIdx.x] =
        first ? make_double2(0.0, 0.0) : make_double2(__ldcg(wst + gi), __ldcg(wst + G + gi));
  }
  for (int p = 0; p < npairs; ++p) {
    const double2 *zs = in + (int64_t)(2 * p) * G + rbase;
    const double2 *ws = zs + G;
    prefetch_pair(in, G, p + 1, npairs, tile * P::NL * P::N, P::NL * P::N);
    double2 z[8], w[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) z[r] = __ldcg(zs + in_pos<LOGN>(t, r));
    tile_fft_reg<LOGN, 1, false, kEL<LOGN>>(smem, z, sm_tw);
#pragma unroll
    for (int r = 0; r < 8; ++r) w[r] = __ldcg(ws + in_pos<LOGN>(t, r));
    tile_fft_reg<LOGN, 1, false, kEL<LOGN>>(smem, w, sm_tw);
    const int b = b0 + 2 * p;
    const double inv_a = recip_of(b + 1), inv_b = recip_of(b + 2);
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
__device__ void means_tile(double2 *smem, double2 *sm_tw, const double2 *in, const double *wst, int64_t G, int nboot,
                           double vscale, double dlogt, double eps, int64_t steps_low, int64_t steps_over,
                           const StepState &cs, int step, int64_t tile) {
  using P = EP<LOGN>;
  using I = TileIdx<LOGN, false, kEL<LOGN>>;
  const int64_t rbase = (tile * P::NL + I::line()) * P::N;
  const int t = I::bfly();
  double2 z[8];
#pragma unroll
  for (int r = 0; r < 8; ++r) z[r] = __ldcg(in + rbase + in_pos<LOGN>(t, r));
  tile_fft_reg<LOGN, 1, false, kEL<LOGN>>(smem, z, sm_tw);
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int64_t gi = rbase + out_pos<LOGN>(t, i);
    const double mu = sqrt(z[i].x * z[i].x + z[i].y * z[i].y);
    const double m2 = __ldcg(wst + G + gi);
    step_update<true>(cs, gi, mu, vscale * m2 / (double)(nboot - 1), dlogt, eps, steps_low, steps_over, step);
  }
}

// ------------------------------------------------- tile bodies, any line length
// The same three tile kinds for axes whose length is not a power of two in 16..2048:
// TL lines staged in shared memory (two buffers of TL x (n + 1)), the Stockham
// mixed-radix FFT of pkde_internal.cuh (radix 8/4/2/3/5, generic odd radix), twiddles
// from the table of the line length.

// Lines L0 .. L0+TL-1 along an axis with stride `inner`; element k of line L sits at
// (L / inner) * n * inner + (L % inner) + k * inner.  Consecutive threads take
// consecutive lines (coalesced wherever adjacent lines are adjacent in memory).
template <bool FROM_SPECTRA>
__device__ void axis_tiles_gen(double2 *smem, const double2 *in, double2 *out, int n, int64_t inner,
                               int64_t first_tile, int ntiles, const double *f, int TL, const FftPlan &plan,
                               const double2 *tw, const EngineEst &E, const PassScale ps) {
  const int pitch = n + 1;
  double2 *bufA = smem, *bufB = smem + TL * pitch;
  // TL is a power of two dividing the block size: thread i always serves line i % TL,
  // elements k = i / TL, i / TL + kstep, ...
  const int l = threadIdx.x & (TL - 1);
  const int kstep = blockDim.x / TL;
  const int k0 = threadIdx.x / TL;
  for (int u = 0; u < ntiles; ++u) {
    const int64_t L = (first_tile + u) * TL + l;
    const int64_t base = (L / inner) * n * inner + (L % inner);
    double cl = 1.0;
    if constexpr (FROM_SPECTRA) cl = line_scale(E, ps, L);
    for (int k = k0; k < n; k += kstep) {
      const int64_t off = base + (int64_t)k * inner;
      if constexpr (FROM_SPECTRA) bufA[l * pitch + k] = cscale(__ldcs(in + off), f[k] * cl);
      else bufA[l * pitch + k] = __ldcg(in + off);
    }
    __syncthreads();
    const double2 *res = smem_fft<1>(bufA, bufB, pitch, TL, plan, tw);
    for (int k = k0; k < n; k += kstep) __stcg(out + base + (int64_t)k * inner, res[l * pitch + k]);
    __syncthreads();
  }
}

// Final pass, TL contiguous rows of length n1 (npts = TL * n1 <= 8 * kEngineThreads):
// inverse FFT of the z and w rows of every pair, VMR of both bootstraps of a pair and
// the Welford update over bootstraps in order (state per point in shared memory).
__device__ void vmr_tile_gen(double2 *smem, double2 *state, const double2 *in, int npairs, int b0, int nboot,
                             double inv_n, int64_t G, double *wst, int first, int64_t tile, int n1, int TL,
                             const FftPlan &plan, const double2 *tw, FastDiv dn1) {
  const int pitch = n1 + 1;
  double2 *bufA = smem, *bufB = smem + TL * pitch;
  const int npts = TL * n1;
  const int64_t rbase = tile * npts;
  prefetch_pair(in, G, 0, npairs, rbase, npts);
  for (int e = threadIdx.x; e < npts; e += blockDim.x)
    state[e] = first ? make_double2(0.0, 0.0) : make_double2(__ldcg(wst + rbase + e), __ldcg(wst + G + rbase + e));
  for (int p = 0; p < npairs; ++p) {
    const double2 *zs = in + (int64_t)(2 * p) * G + rbase;
    const double2 *ws = zs + G;
    prefetch_pair(in, G, p + 1, npairs, rbase, npts);
    double2 zval[8];
    for (int e = threadIdx.x; e < npts; e += blockDim.x) {
      const int l = (int)fdiv((uint32_t)e, dn1), k = e - l * n1;
      bufA[l * pitch + k] = __ldcg(zs + e);
    }
    __syncthreads();
    const double2 *rz = smem_fft<1>(bufA, bufB, pitch, TL, plan, tw);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = threadIdx.x + q * kEngineThreads;
      if (e < npts) zval[q] = rz[e + (int)fdiv((uint32_t)e, dn1) * (pitch - n1)];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < npts; e += blockDim.x) {
      const int l = (int)fdiv((uint32_t)e, dn1), k = e - l * n1;
      bufA[l * pitch + k] = __ldcg(ws + e);
    }
    __syncthreads();
    const double2 *rw = smem_fft<1>(bufA, bufB, pitch, TL, plan, tw);
    const int b = b0 + 2 * p;
    const double inv_a = recip_of(b + 1), inv_b = recip_of(b + 2);
    const bool has_b = b + 1 < nboot;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = threadIdx.x + q * kEngineThreads;
      if (e < npts) {
        const double2 w = rw[e + (int)fdiv((uint32_t)e, dn1) * (pitch - n1)];
        double2 st = state[e];
        welford(vmr_of(zval[q].x, w.x, inv_n), inv_a, st.x, st.y);
        if (has_b) welford(vmr_of(zval[q].y, w.y, inv_n), inv_b, st.x, st.y);
        state[e] = st;
      }
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < npts; e += blockDim.x) {
    const double2 st = state[e];
    __stcg(wst + rbase + e, st.x);
    __stcg(wst + G + rbase + e, st.y);
  }
}

__device__ void means_tile_gen(double2 *smem, const double2 *in, const double *wst, int64_t G, int nboot,
                               double vscale, double dlogt, double eps, int64_t steps_low, int64_t steps_over,
                               const StepState &cs, int step, int64_t tile, int n1, int TL, const FftPlan &plan,
                               const double2 *tw, FastDiv dn1) {
  const int pitch = n1 + 1;
  double2 *bufA = smem, *bufB = smem + TL * pitch;
  const int npts = TL * n1;
  const int64_t rbase = tile * npts;
  for (int e = threadIdx.x; e < npts; e += blockDim.x) {
    const int l = (int)fdiv((uint32_t)e, dn1), k = e - l * n1;
    bufA[l * pitch + k] = __ldcg(in + rbase + e);
  }
  __syncthreads();
  const double2 *res = smem_fft<1>(bufA, bufB, pitch, TL, plan, tw);
  for (int e = threadIdx.x; e < npts; e += blockDim.x) {
    const double2 z = res[e + (int)fdiv((uint32_t)e, dn1) * (pitch - n1)];
    const int64_t gi = rbase + e;
    const double mu = sqrt(z.x * z.x + z.y * z.y);
    const double m2 = __ldcg(wst + G + gi);
    step_update<true>(cs, gi, mu, vscale * m2 / (double)(nboot - 1), dlogt, eps, steps_low, steps_over, step);
  }
}

// ------------------------------------------------- tile bodies, N = R * 2^LM
// Axes of N = R * M points (R = 3 or 5, M = 2^LM, 8 <= M <= 256): the line splits into
// R interleaved sub-lines x[R*n2 + n1] of M points; each goes through the register
// radix-8 FFT (one butterfly per thread, column mapping over all sub-lines of the tile),
// then a radix-R combine per output pair: X[k2 + M*q] = sum_n1 W_N^(n1*k2) Y_n1[k2]
// W_R^(n1*q) (decimation in time at the top level).  The M-point results pass through the
// tile (same padded layout) to the combine threads.
__host__ __device__ constexpr int p2floor(int x) { return x < 2 ? 1 : 2 * p2floor(x / 2); }

template <int R, int LM>
struct Mix {
  static constexpr int M = 1 << LM;
  static constexpr int N = R * M;
  static constexpr int NB8 = M / 8;
  static constexpr int NLA = p2floor(kEngineThreads / (R * NB8));  // lines per axis-pass tile
  static constexpr int NLF = NLA > 1 ? NLA / 2 : 1;                 // rows per final-pass tile
  static_assert(2 * R * NLF * NB8 <= kEngineThreads, "final-pass tile exceeds the block");
};

// Geometry of one tile: A arrays (1: axis and means passes; 2: z and w of the VMR pass)
// of NL lines, each line R sub-lines of M points.  Sub-line sub = (a R + n1) NL + l.
template <int R, int LM, int NL, int A>
struct MixTile {
  using X = Mix<R, LM>;
  static constexpr int SUB = A * R * NL;
  static constexpr int FT = SUB * X::NB8;                           // threads in the M-point FFTs
  static constexpr int LPAD = pad8(X::M);
  static constexpr int LP = LPAD + ((1 - (LPAD % 8)) % 8 + 8) % 8;  // sub-line pitch, 1 mod 8
  static constexpr int TILE = (SUB + 1) * LP;                       // + a scratch sub-line for idle threads
  static constexpr int ITEMS = NL * X::M;                           // combine items (per array)
  static constexpr int PER = (ITEMS + kEngineThreads - 1) / kEngineThreads;
};

// The calling thread's role in the M-point FFTs: sub-line (array a, phase n1, line l)
// and butterfly t; threads beyond FT run the scratch sub-line.
template <class T>
struct MixRole {
  bool act;
  int sub, t, a, n1, l;
  __device__ __forceinline__ MixRole() {
    const int tid = threadIdx.x;
    act = tid < T::FT;
    sub = act ? tid % T::SUB : T::SUB;
    t = act ? tid / T::SUB : (tid - T::FT) % T::X::NB8;
    constexpr int nl = T::ITEMS / T::X::M;
    constexpr int R = T::X::N / T::X::M;
    l = sub % nl;
    n1 = (sub / nl) % R;
    a = sub / (nl * R);
  }
};

// M-point FFTs of the tile's sub-lines (v: the thread's 8 scaled inputs of line positions
// R * in_pos(t, r) + n1), results into the tile for the combine.  All threads call.
template <class T>
__device__ __forceinline__ void mix_fft(double2 *tile, const double2 *sm_tw, const MixRole<T> &ro, double2 (&v)[8]) {
  constexpr int LM = cilog2(T::X::M);
  run_stages<LM, 1, 0, true, 0>(tile + ro.sub * T::LP, nullptr, v, ro.t, sm_tw, 0);
  if (ro.act) {
#pragma unroll
    for (int i = 0; i < 8; ++i) tile[ro.sub * T::LP + pad8(out_pos<LM>(ro.t, i))] = v[i];
  }
  __syncthreads();
}

// Combine item `it` of the thread for array a: y[q] = X[k2 + M q] of line
// threadIdx.x % NL.  Returns false when the thread has no such item.
template <class T>
__device__ __forceinline__ bool mix_combine(const double2 *tile, const double2 *twc, int it, int a, int &k2,
                                            double2 (&y)[T::X::N / T::X::M]) {
  constexpr int R = T::X::N / T::X::M;
  constexpr int NL = T::ITEMS / T::X::M;
  const int idx = threadIdx.x + it * kEngineThreads;
  if (idx >= T::ITEMS) return false;
  const int l = idx % NL;
  k2 = idx / NL;
#pragma unroll
  for (int n1 = 0; n1 < R; ++n1) {
    double2 v = tile[((a * R + n1) * NL + l) * T::LP + pad8(k2)];
    if (n1 > 0) v = cmul(v, __ldg(twc + (n1 - 1) * T::X::M + k2));
    y[n1] = v;
  }
  if constexpr (R == 3) dft3<1>(y);
  else dft5<1>(y);
  return true;
}

// The three mixed-radix tile bodies are separate (not inlined) functions: inlined into the
// persistent kernel beside every other (R, M) instantiation they shared its 128 registers
// with the item loop's live values and spilled (1.4 KB of stack); compiled on their own
// they spill nothing (96^3 1.22 -> 1.09 ns per grid-point step, 80^3 1.50 -> 1.14).
template <int R, int LM, bool FROM_SPECTRA>
__device__ __noinline__ void axis_tiles_mix(double2 *tile, const double2 *sm_tw, const double2 *twc, const double2 *in,
                               double2 *out, int64_t inner, int64_t first_tile, int ntiles, const double *f,
                               const EngineEst &E, const PassScale ps) {
  using X = Mix<R, LM>;
  using T = MixTile<R, LM, X::NLA, 1>;
  const MixRole<T> ro;
  const int lc = threadIdx.x % X::NLA;  // the combine line (NLA divides the block)
  // With `inner` a multiple of NLA a tile's lines are adjacent in memory: N segments of
  // NLA * 16 contiguous bytes, which are brought into L2 for the next tile while this one
  // is transformed (as in the power-of-two column passes).
  const bool pf = inner % X::NLA == 0;
  for (int u = 0; u < ntiles; ++u) {
    const int64_t L0 = (first_tile + u) * X::NLA;
    const int64_t Lf = L0 + ro.l, Lc = L0 + lc;
    const int64_t bf = (Lf / inner) * X::N * inner + (Lf % inner);
    const int64_t bc = (Lc / inner) * X::N * inner + (Lc % inner);
    double2 v[8];
    double cl = 1.0;
    if constexpr (FROM_SPECTRA) cl = line_scale(E, ps, Lf);
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int pos = R * in_pos<LM>(ro.t, r) + ro.n1;
      const int64_t off = bf + (int64_t)pos * inner;
      if constexpr (FROM_SPECTRA) v[r] = ro.act ? cscale(__ldcs(in + off), f[pos] * cl) : make_double2(0.0, 0.0);
      else v[r] = ro.act ? __ldcg(in + off) : make_double2(0.0, 0.0);
    }
    if (pf && u + 1 < ntiles) {
      const int64_t Ln = L0 + X::NLA;  // first line of the next tile (Ln % inner + NLA <= inner)
      const double2 *b0 = in + (Ln / inner) * X::N * inner + (Ln % inner);
      for (int k = threadIdx.x; k < X::N; k += kEngineThreads)
        prefetch_l2(b0 + (int64_t)k * inner, (uint32_t)(X::NLA * sizeof(double2)));
    }
    mix_fft<T>(tile, sm_tw, ro, v);
#pragma unroll
    for (int it = 0; it < T::PER; ++it) {
      int k2;
      double2 y[R];
      if (mix_combine<T>(tile, twc, it, 0, k2, y)) {
#pragma unroll
        for (int q = 0; q < R; ++q) __stcg(out + bc + (int64_t)(k2 + X::M * q) * inner, y[q]);
      }
    }
    __syncthreads();
  }
}

// Final pass: NLF rows; the tile holds the z and the w sub-lines of those rows, so each
// combine item has both transforms of its points for the VMR and the Welford update.
template <int R, int LM>
__device__ __noinline__ void vmr_tile_mix(double2 *tile, double2 *state, const double2 *sm_tw, const double2 *twc,
                             const double2 *in, int npairs, int b0, int nboot, double inv_n, int64_t G, double *wst,
                             int first, int64_t tile_idx) {
  using X = Mix<R, LM>;
  using T = MixTile<R, LM, X::NLF, 2>;
  const MixRole<T> ro;
  const int npts = X::NLF * X::N;
  const int64_t rbase = tile_idx * npts;
  // The Welford state sits in shared memory in combine-item order: entry q ITEMS + idx is
  // point (row idx % NLF, position idx / NLF + M q) of the tile, so consecutive threads
  // update consecutive entries.  (In point order their rows lie N apart, and N = R M with
  // M >= 8 is a multiple of 8 16-byte units: every access an 8-way bank conflict.)
  auto point_of = [](int si) {
    const int q = si / T::ITEMS, idx = si - q * T::ITEMS;
    return (idx % X::NLF) * X::N + idx / X::NLF + X::M * q;
  };
  prefetch_pair(in, G, 0, npairs, rbase, npts);
  for (int si = threadIdx.x; si < npts; si += blockDim.x) {
    const int e = point_of(si);
    state[si] = first ? make_double2(0.0, 0.0) : make_double2(__ldcg(wst + rbase + e), __ldcg(wst + G + rbase + e));
  }
  for (int p = 0; p < npairs; ++p) {
    prefetch_pair(in, G, p + 1, npairs, rbase, npts);
    const double2 *src = in + (int64_t)(2 * p + ro.a) * G + rbase + ro.l * X::N;
    double2 v[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int pos = R * in_pos<LM>(ro.t, r) + ro.n1;
      v[r] = ro.act ? __ldcg(src + pos) : make_double2(0.0, 0.0);
    }
    mix_fft<T>(tile, sm_tw, ro, v);
    const int b = b0 + 2 * p;
    const double inv_a = recip_of(b + 1), inv_b = recip_of(b + 2);
    const bool has_b = b + 1 < nboot;
#pragma unroll
    for (int it = 0; it < T::PER; ++it) {
      int k2;
      double2 z[R], w[R];
      if (mix_combine<T>(tile, twc, it, 0, k2, z)) {
        mix_combine<T>(tile, twc, it, 1, k2, w);
        const int idx = threadIdx.x + it * kEngineThreads;  // the combine item (k2 = idx / NLF)
#pragma unroll
        for (int q = 0; q < R; ++q) {
          double2 st = state[q * T::ITEMS + idx];
          welford(vmr_of(z[q].x, w[q].x, inv_n), inv_a, st.x, st.y);
          if (has_b) welford(vmr_of(z[q].y, w[q].y, inv_n), inv_b, st.x, st.y);
          state[q * T::ITEMS + idx] = st;
        }
      }
    }
    __syncthreads();
  }
  for (int si = threadIdx.x; si < npts; si += blockDim.x) {
    const int e = point_of(si);
    const double2 st = state[si];
    __stcg(wst + rbase + e, st.x);
    __stcg(wst + G + rbase + e, st.y);
  }
}

// Means pass over the same NLF rows (one array; the second array's threads idle).
template <int R, int LM>
__device__ __noinline__ void means_tile_mix(double2 *tile, const double2 *sm_tw, const double2 *twc, const double2 *in,
                               const double *wst, int64_t G, int nboot, double vscale, double dlogt, double eps,
                               int64_t steps_low, int64_t steps_over, const StepState &cs, int step,
                               int64_t tile_idx) {
  using X = Mix<R, LM>;
  using T = MixTile<R, LM, X::NLF, 1>;
  const MixRole<T> ro;
  const int64_t rbase = tile_idx * (X::NLF * X::N);
  const int lrow = (threadIdx.x % X::NLF) * X::N;
  const double2 *src = in + rbase + ro.l * X::N;
  double2 v[8];
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int pos = R * in_pos<LM>(ro.t, r) + ro.n1;
    v[r] = ro.act ? __ldcg(src + pos) : make_double2(0.0, 0.0);
  }
  mix_fft<T>(tile, sm_tw, ro, v);
#pragma unroll
  for (int it = 0; it < T::PER; ++it) {
    int k2;
    double2 y[R];
    if (mix_combine<T>(tile, twc, it, 0, k2, y)) {
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const int64_t gi = rbase + lrow + k2 + X::M * q;
        const double mu = sqrt(y[q].x * y[q].x + y[q].y * y[q].y);
        const double m2 = __ldcg(wst + G + gi);
        step_update<true>(cs, gi, mu, vscale * m2 / (double)(nboot - 1), dlogt, eps, steps_low, steps_over, step);
      }
    }
  }
  __syncthreads();
}

#define PKDE_MIX_SWITCH(R, LM, CALL)                                                     \
  if (R == 3) {                                                                          \
    switch (LM) {                                                                        \
      case 3: CALL(3, 3); break;                                                         \
      case 4: CALL(3, 4); break;                                                         \
      case 5: CALL(3, 5); break;                                                         \
      case 6: CALL(3, 6); break;                                                         \
      case 7: CALL(3, 7); break;                                                         \
      case 8: CALL(3, 8); break;                                                         \
      default: break;                                                                    \
    }                                                                                    \
  } else {                                                                               \
    switch (LM) {                                                                        \
      case 3: CALL(5, 3); break;                                                         \
      case 4: CALL(5, 4); break;                                                         \
      case 5: CALL(5, 5); break;                                                         \
      case 6: CALL(5, 6); break;                                                         \
      case 7: CALL(5, 7); break;                                                         \
      default: break;                                                                    \
    }                                                                                    \
  }

// ------------------------------------------------------------------ the engine
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

// GEN: some estimation of the launch has an axis on the shared-memory FFT path (a
// separate instantiation keeps the register pressure of all-power-of-two launches low).
template <bool GEN>
__global__ void __launch_bounds__(kEngineThreads, kEngineCtas) engine_kernel(EngineRun R, int max_tile,
                                                                             int state_elems) {
  extern __shared__ double2 smem[];
  // [tile][state: Welford state of the final pass, second exchange buffer of the axis
  // passes][twiddles]
  double2 *tile_mem = smem;
  double2 *state = smem + max_tile;
  double2 *sm_tw = state + state_elems;
  __shared__ EngineEst sE;  // descriptor of the estimation the current item belongs to
  __shared__ int64_t s_next, s_b, s_tile, s_round, s_off;
  __shared__ int s_p, s_ok, s_e;
  int cached_tw = -1;
  int cached_e = -1;
  int64_t cur = 0;  // segment cursor (warp 0; items of a CTA increase, so it only moves forward)
  // The next item is taken while the current one runs (items are taken in increasing
  // order per CTA, so every wait still points to an earlier item).
  if (threadIdx.x == 0) s_next = (int64_t)atomicAdd(R.next, 1);
  __syncthreads();
  int64_t item = s_next;
  for (;;) {
    if (item >= R.total_items) break;
    __syncthreads();  // everyone has read s_next and finished with sE
    if (threadIdx.x == 0) s_next = ld_acquire(R.error) ? R.total_items : (int64_t)atomicAdd(R.next, 1);
    // ---- segment of `item`: seg_start is increasing, so the lanes whose entry is
    // <= item form a prefix; advance by its length (32 entries per iteration)
    if (threadIdx.x < 32) {
      for (;;) {
        const int64_t k = cur + 1 + threadIdx.x;
        const bool le = k <= R.nseg && __ldg(R.seg_start + k) <= item;
        const int c = __popc(__ballot_sync(0xffffffffu, le));
        cur += c;
        if (c < 32) break;
      }
      if (threadIdx.x == 0) {
        const int2 sg = __ldg(R.seg + cur);
        s_e = sg.x;
        s_round = sg.y;
        s_off = item - __ldg(R.seg_start + cur);
      }
    }
    __syncthreads();
    if (s_e != cached_e) {
      cached_e = s_e;
      const int *src = reinterpret_cast<const int *>(R.est + cached_e);
      int *dst = reinterpret_cast<int *>(&sE);
      for (int i = threadIdx.x; i < (int)(sizeof(EngineEst) / sizeof(int)); i += blockDim.x) dst[i] = __ldg(src + i);
      __syncthreads();
    }
    const EngineEst &E = sE;
    // ---- decode (thread 0) and dependencies (thread 0 spins; acquire orders the data
    // reads after it)
    if (threadIdx.x == 0) {
      bool ok = false;
      int64_t off = s_off;
      for (int p = E.P - 1; p >= 0; --p) {
        const int64_t b = s_round - (int64_t)p * E.D;
        if (b < 0 || b >= E.NB) continue;
        const int n = pass_tiles(E, b, p);
        if (off < n) {
          s_b = b;
          s_p = p;
          s_tile = off;
          ok = true;
          break;
        }
        off -= n;
      }
      if (ok) {
        const int64_t b = s_b;
        const int p = s_p;
        const int64_t s = b / (E.J + 1);
        const int j = (int)(b % (E.J + 1));
        if (p == 0) {
          if (b >= E.Q) ok = wait_geq(R.error, E.cnt + (b - E.Q) * E.P + (E.P - 1), pass_tiles(E, b - E.Q, E.P - 1), R.spin_limit);
        } else {
          ok = wait_geq(R.error, E.cnt + b * E.P + (p - 1), pass_tiles(E, b, p - 1), R.spin_limit);
        }
        if (ok && p == E.P - 1) {
          if (j > 0) ok = wait_geq(R.error, E.fin + (b - 1) * E.Tf + s_tile, 1, R.spin_limit);  // Welford order / all groups done
          if (ok && j == 0 && s >= 2)                                                // state slot free
            ok = wait_geq(R.error, E.fin + ((s - 2) * (E.J + 1) + E.J) * E.Tf + s_tile, 1, R.spin_limit);
          if (ok && j == E.J && s >= 1)                                              // convergence order
            ok = wait_geq(R.error, E.fin + ((s - 1) * (E.J + 1) + E.J) * E.Tf + s_tile, 1, R.spin_limit);
        }
      } else {
        atomicExch(R.error, 1);  // the schedule and the descriptor disagree
      }
      s_ok = ok;
    }
    __syncthreads();
    if (!s_ok) break;
    const int64_t b = s_b;
    const int p = s_p;
    const int64_t tile = s_tile;
    const int64_t s = b / (E.J + 1);
    const int j = (int)(b % (E.J + 1));
    const bool means = j == E.J;
    const int64_t slot = b % E.Q;
    double2 *slot_base = E.slots + slot * E.slot_elems;
    // ---- work
    const double *fzs = E.fz + s * E.tab_stride;
    const double *fws = E.fw + s * E.tab_stride;
    if (p < E.P - 1) {
      const int a = E.ndim - 1 - p;
      const int ln = E.logn[a];
      const int64_t lines = E.G / E.dims[a];
      const int tpi = E.tpi[a];
      const int64_t ipa = lines / ((int64_t)E.tl[a] * tpi);  // items per array
      const int64_t arr = tile / ipa;
      const int64_t first_tile = (tile % ipa) * tpi;
      int64_t inner = 1;
      for (int q = 0; q < a; ++q) inner *= E.dims[q];
      const double2 *in = p == 0 ? (means ? E.spectra + (int64_t)(2 * E.npairs) * E.G
                                          : E.spectra + (int64_t)(2 * j * E.g) * E.G)
                                 : slot_base;
      in += arr * E.G;
      double2 *out = slot_base + arr * E.G;
      // pass 0: the line's own axis factor per element, every other factor and the array's
      // scalar per line (PassScale); later passes apply nothing
      const bool second = !means && (arr & 1);
      const double *f = (second ? fws : fzs) + E.aoff[a];
      const PassScale ps{second ? fws : fzs, second ? E.invG * E.cw[s] : E.invG};
#define PKDE_AXIS(L)                                                                             \
  {                                                                                              \
    stage_tw<L>(sm_tw, R.tw[L], cached_tw, L);                                                   \
    if (p == 0)                                                                                  \
      axis_tiles<L, true>(tile_mem, state, sm_tw, in, out, inner, first_tile, tpi, f, E, ps);    \
    else                                                                                         \
      axis_tiles<L, false>(tile_mem, state, sm_tw, in, out, inner, first_tile, tpi, f, E, ps);   \
  }
#define PKDE_AXIS_MIX(RR, LL)                                                                             \
  {                                                                                                       \
    stage_tw<LL>(sm_tw, R.tw[LL], cached_tw, LL);                                                         \
    if (p == 0)                                                                                           \
      axis_tiles_mix<RR, LL, true>(tile_mem, sm_tw, E.twc[a], in, out, inner, first_tile, tpi, f, E, ps);  \
    else                                                                                                  \
      axis_tiles_mix<RR, LL, false>(tile_mem, sm_tw, E.twc[a], in, out, inner, first_tile, tpi, f, E, ps); \
  }
      if (GEN && E.gen[a] == 1) {
        if (p == 0)
          axis_tiles_gen<true>(tile_mem, in, out, (int)E.dims[a], inner, first_tile, tpi, f, E.tl[a], E.plan[a],
                               E.twg[a], E, ps);
        else
          axis_tiles_gen<false>(tile_mem, in, out, (int)E.dims[a], inner, first_tile, tpi, f, E.tl[a], E.plan[a],
                                E.twg[a], E, ps);
      } else if (GEN && E.gen[a] == 2) {
        PKDE_MIX_SWITCH(E.mixr[a], ln, PKDE_AXIS_MIX)
      } else {
        PKDE_ENGINE_SWITCH(ln, PKDE_AXIS)
      }
#undef PKDE_AXIS
#undef PKDE_AXIS_MIX
    } else {
      const int ln = E.logn[0];
      if (!means) {
        const int np = batch_arrays(E, b) / 2;
#define PKDE_VMR(L)                                                                                         \
  {                                                                                                         \
    stage_tw<L>(sm_tw, R.tw[L], cached_tw, L);                                                              \
    vmr_tile<L>(tile_mem, state, sm_tw, slot_base, np, 2 * j * E.g, E.nboot, E.inv_n, E.G,                  \
                E.wstate + (s & 1) * 2 * E.G, j == 0, tile);                                                \
  }
#define PKDE_VMR_MIX(RR, LL)                                                                              \
  {                                                                                                       \
    stage_tw<LL>(sm_tw, R.tw[LL], cached_tw, LL);                                                         \
    vmr_tile_mix<RR, LL>(tile_mem, state, sm_tw, E.twc[0], slot_base, np, 2 * j * E.g, E.nboot, E.inv_n,   \
                         E.G, E.wstate + (s & 1) * 2 * E.G, j == 0, tile);                                 \
  }
        if (GEN && E.gen[0] == 2) {
          PKDE_MIX_SWITCH(E.mixr[0], ln, PKDE_VMR_MIX)
        } else if (GEN && E.gen[0]) {
          vmr_tile_gen(tile_mem, state, slot_base, np, 2 * j * E.g, E.nboot, E.inv_n, E.G,
                       E.wstate + (s & 1) * 2 * E.G, j == 0, tile, (int)E.dims[0], E.tl[0], E.plan[0], E.twg[0],
                       E.dlen[0]);
        } else {
          PKDE_ENGINE_SWITCH(ln, PKDE_VMR)
        }
#undef PKDE_VMR
#undef PKDE_VMR_MIX
      } else {
#define PKDE_MEANS(L)                                                                                        \
  {                                                                                                          \
    stage_tw<L>(sm_tw, R.tw[L], cached_tw, L);                                                               \
    means_tile<L>(tile_mem, sm_tw, slot_base, E.wstate + (s & 1) * 2 * E.G, E.G, E.nboot, E.vscale[s],        \
                  E.dlogt[s], E.eps, E.steps_low, E.steps_over, E.cs, (int)s, tile);                         \
  }
#define PKDE_MEANS_MIX(RR, LL)                                                                          \
  {                                                                                                     \
    stage_tw<LL>(sm_tw, R.tw[LL], cached_tw, LL);                                                       \
    means_tile_mix<RR, LL>(tile_mem, sm_tw, E.twc[0], slot_base, E.wstate + (s & 1) * 2 * E.G, E.G,      \
                           E.nboot, E.vscale[s], E.dlogt[s], E.eps, E.steps_low, E.steps_over, E.cs,     \
                           (int)s, tile);                                                                \
  }
        if (GEN && E.gen[0] == 2) {
          PKDE_MIX_SWITCH(E.mixr[0], ln, PKDE_MEANS_MIX)
        } else if (GEN && E.gen[0]) {
          means_tile_gen(tile_mem, slot_base, E.wstate + (s & 1) * 2 * E.G, E.G, E.nboot, E.vscale[s], E.dlogt[s],
                         E.eps, E.steps_low, E.steps_over, E.cs, (int)s, tile, (int)E.dims[0], E.tl[0], E.plan[0],
                         E.twg[0], E.dlen[0]);
        } else {
          PKDE_ENGINE_SWITCH(ln, PKDE_MEANS)
        }
#undef PKDE_MEANS
#undef PKDE_MEANS_MIX
      }
    }
    // ---- signal completion
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      if (p == E.P - 1) add_release(E.fin + b * E.Tf + tile, 1);
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
  case L: return EP<L>::TILE;
    PKDE_T(4) PKDE_T(5) PKDE_T(6) PKDE_T(7) PKDE_T(8) PKDE_T(9) PKDE_T(10) PKDE_T(11)
#undef PKDE_T
    default: return 0;
  }
}
size_t tw_elems(int logn) {
  switch (logn) {
#define PKDE_T(L) \
  case L: return EP<L>::TWSIZE;
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

#define PKDE_MIX_HOST(RR, LL) return fn(Mix<RR, LL>{});
template <class F>
static size_t mix_dispatch(int R, int lm, F fn) {
  PKDE_MIX_SWITCH(R, lm, PKDE_MIX_HOST)
  return 0;
}
#undef PKDE_MIX_HOST
// lines per tile: axis passes (axis >= 2) and the final pass (axis 1)
static int mix_lines(int R, int lm, bool final_pass) {
  return (int)mix_dispatch(R, lm, [&](auto x) { return (size_t)(final_pass ? decltype(x)::NLF : decltype(x)::NLA); });
}
static size_t mix_tile_elems(int R, int lm) {
  return mix_dispatch(R, lm, [](auto x) {
    using X = decltype(x);
    constexpr int R_ = X::N / X::M, LM_ = cilog2(X::M);
    return std::max<size_t>({MixTile<R_, LM_, X::NLA, 1>::TILE, MixTile<R_, LM_, X::NLF, 2>::TILE,
                             MixTile<R_, LM_, X::NLF, 1>::TILE});
  });
}

// Combine twiddles of N = R * M: (cos, sin)(2 pi n1 k2 / N), n1 = 1..R-1, k2 < M.
static const double2 *combine_twiddles_device(pkde_ctx *ctx, int R, int M) {
  const int N = R * M;
  const int key = -(1000000 + 10 * N + R);
  auto it = ctx->twiddles.find(key);
  if (it != ctx->twiddles.end()) return it->second.as<double2>();
  std::vector<double2> tw;
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int n1 = 1; n1 < R; ++n1)
    for (int k2 = 0; k2 < M; ++k2) {
      const long double a = two_pi * (long double)((n1 * k2) % N) / (long double)N;
      tw.push_back(make_double2((double)cosl(a), (double)sinl(a)));
    }
  DevBuf &b = ctx->twiddles[key];
  b.ensure(sizeof(double2) * tw.size());
  PKDE_CUDA_TRY(cudaMemcpy(b.ptr, tw.data(), sizeof(double2) * tw.size(), cudaMemcpyHostToDevice));
  return b.as<double2>();
}

// Tile shape of grid axis j: the register radix-8 FFT where the axis is a power of two
// in 16..8*kEngineThreads whose tiles line up with the layout; otherwise the
// shared-memory mixed-radix FFT for lengths up to 8*kEngineThreads, TL lines per tile
// (a power of two dividing the number of lines, TL x n <= 8*kEngineThreads).
struct AxisShape {
  bool ok;
  int gen;
  int tl;
};
static AxisShape axis_shape(const pkde_grid *g, int j) {
  const int64_t G = grid_size(g);
  int64_t inner = 1;
  for (int q = 0; q < j; ++q) inner *= g->dims[q];
  const int64_t n = g->dims[j];
  const int64_t lines = G / n;
  const int ln = ilog2_pow2(n);
  if (ln >= 4 && (int64_t(1) << ln) <= 8 * kEngineThreads) {
    const int nl = tile_lines_of(ln);
    if (lines % nl == 0 && (j == 0 || inner % nl == 0)) return AxisShape{true, 0, nl};
  }
  // N = R * 2^LM, R = 3 or 5, M = 2^LM in 8..256 (R = 3) or 8..128 (R = 5): mixed-radix
  // register tiles when their lines per tile divide the number of lines
  for (int R : {3, 5}) {
    if (n % R) continue;
    const int lm = ilog2_pow2(n / R);
    if (lm < 3 || lm > (R == 3 ? 8 : 7)) continue;
    const int nl = mix_lines(R, lm, j == 0);
    if (lines % nl == 0) return AxisShape{true, 2, nl};
  }
  if (n < 2 || n > 8 * kEngineThreads) return AxisShape{false, 0, 0};
  int tl = 1;
  const int64_t cap = std::min<int64_t>(16, 8 * kEngineThreads / n);
  while (tl * 2 <= cap && lines % (tl * 2) == 0) tl *= 2;
  return AxisShape{true, 1, tl};
}

bool engine_ok(const pkde_grid *g) {
  if (g->ndim < 2) return false;
  for (int j = 0; j < g->ndim; ++j)
    if (!axis_shape(g, j).ok) return false;
  return true;
}

bool engine_register_only(const pkde_grid *g) {
  for (int j = 0; j < g->ndim; ++j)
    if (axis_shape(g, j).gen) return false;
  return true;
}

namespace {

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Host-side descriptor of one estimation (device pointers filled in later).
EngineEst describe(const EngineArgs &A) {
  const pkde_grid *g = A.grid;
  EngineEst E{};
  E.ndim = g->ndim;
  E.G = grid_size(g);
  for (int j = 0; j < g->ndim; ++j) {
    const AxisShape sh = axis_shape(g, j);
    E.dims[j] = g->dims[j];
    E.gen[j] = sh.gen;
    E.tl[j] = sh.tl;
    E.mixr[j] = 0;
    if (sh.gen == 2) {
      E.mixr[j] = g->dims[j] % 3 == 0 && ilog2_pow2(g->dims[j] / 3) >= 3 ? 3 : 5;
      E.logn[j] = ilog2_pow2(g->dims[j] / E.mixr[j]);
    } else {
      E.logn[j] = sh.gen ? -1 : ilog2_pow2(g->dims[j]);
    }
    E.aoff[j] = A.aoff[j];
  }
  E.npairs = A.npairs;
  E.nboot = A.nboot;
  E.S = A.S;
  E.P = g->ndim;
  // pairs per group: ring slot (2g arrays) within 32 MB, at least one pair.  Larger
  // groups mean fewer, wider batches (more independent tiles per round); measured on
  // 512 x 512 / B = 64: 74 ms at 8 MB, 58.6 ms at 16 MB, 56.9 ms at 32 MB.
  const int64_t arr_bytes = (int64_t)sizeof(double2) * E.G;
  const int64_t slot_mb = A.tune_slot_mb > 0 ? A.tune_slot_mb : engine_env_int("PKDE_ENGINE_SLOT_MB", 32, 1, 256);
  E.g = (int)std::max<int64_t>(1, std::min<int64_t>(E.npairs, (slot_mb << 20) / (2 * arr_bytes)));
  E.J = (E.npairs + E.g - 1) / E.g;
  // pipeline delay between passes of one batch; ring slots cover the delay
  E.D = A.tune_delay > 0 ? A.tune_delay : engine_env_int("PKDE_ENGINE_DELAY", 2, 1, 8);
  // ring slots: the pipeline depth plus a margin (extra slots let pass 0 of a batch start
  // before the final pass of the batch Q earlier has released its slot)
  E.Q = (E.P - 1) * E.D + 2 + (A.tune_qextra > 0 ? A.tune_qextra : engine_env_int("PKDE_ENGINE_QEXTRA", 0, 0, 8));
  E.NB = (int64_t)E.S * (E.J + 1);
  E.Tf = (int)((E.G / E.dims[0]) / E.tl[0]);
  for (int a = 0; a < 4; ++a) E.tpi[a] = 1;
  for (int a = 1; a < E.ndim; ++a) {
    const int64_t tiles = (E.G / E.dims[a]) / E.tl[a];
    // tiles per axis-pass item: 2 for 2-D, 8 for 3-D/4-D (measured on 128^3 / B = 32:
    // 300 ms at 2, 267 ms at 4, 246 ms at 8)
    int want = A.tune_tpi > 0 ? A.tune_tpi : engine_env_int("PKDE_ENGINE_TPI", E.ndim == 2 ? 2 : 8, 1, 16);
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
  return E;
}

}  // namespace

void run_engine_batch(pkde_ctx *ctx, const EngineArgs *args, int count, cudaStream_t st) {
  if (count < 1) return;
  if (!ctx->recip_ready) {
    std::vector<double> r(kRecip, 0.0);
    for (int i = 1; i < kRecip; ++i) r[i] = 1.0 / (double)i;
    PKDE_CUDA_TRY(cudaMemcpyToSymbol(c_recip, r.data(), sizeof(double) * kRecip));
    ctx->recip_ready = true;
  }
  std::vector<EngineEst> est(count);
  std::vector<std::array<FftPlan, 4>> plans(count);
  std::vector<std::vector<int64_t>> rs(count);
  size_t max_tile = 0, max_tw = 1, max_reg_tile = 0;
  EngineRun R{};
  for (int l = 0; l < 13; ++l) R.tw[l] = nullptr;
  for (int e = 0; e < count; ++e) {
    EngineEst &E = est[e];
    E = describe(args[e]);
    for (int j = 0; j < E.ndim; ++j) {
      if (E.gen[j] == 2) {
        R.tw[E.logn[j]] = stage_twiddles_device(ctx, E.logn[j]);
        E.twc[j] = combine_twiddles_device(ctx, E.mixr[j], 1 << E.logn[j]);
        max_tile = std::max(max_tile, mix_tile_elems(E.mixr[j], E.logn[j]));
        max_tw = std::max(max_tw, tw_elems(E.logn[j]));
      } else if (E.gen[j]) {
        E.twg[j] = twiddles_device(ctx, (int)E.dims[j]);
        plans[e][j] = make_plan((int)E.dims[j]);
        E.dlen[j] = make_fastdiv((uint32_t)E.dims[j]);
        max_tile = std::max(max_tile, (size_t)2 * E.tl[j] * (size_t)(E.dims[j] + 1));
      } else {
        R.tw[E.logn[j]] = stage_twiddles_device(ctx, E.logn[j]);
        max_tile = std::max(max_tile, tile_elems(E.logn[j]));
        max_reg_tile = std::max(max_reg_tile, tile_elems(E.logn[j]));
        max_tw = std::max(max_tw, tw_elems(E.logn[j]));
      }
    }
    // local schedule: items per round
    std::vector<int64_t> &r = rs[e];
    r.assign(E.nrounds + 1, 0);
    for (int64_t k = 0; k < E.nrounds; ++k) {
      int64_t n = 0;
      for (int p = 0; p < E.P; ++p) {
        const int64_t b = k - (int64_t)p * E.D;
        if (b >= 0 && b < E.NB) n += pass_tiles(E, b, p);
      }
      r[k + 1] = r[k] + n;
    }
  }
  // Global schedule.  Estimations are dealt to `lanes` lanes in order (each to the lane
  // that frees first); a lane runs its estimations one after another, lanes run side by
  // side.  More lanes: more independent work per round; fewer: a smaller working set.
  const int lanes = engine_env_int("PKDE_ENGINE_LANES", count, 1, 1 << 20);
  std::vector<int64_t> start(count), lane_end(std::min(lanes, count), 0);
  for (int e = 0; e < count; ++e) {
    size_t best = 0;
    for (size_t l = 1; l < lane_end.size(); ++l)
      if (lane_end[l] < lane_end[best]) best = l;
    start[e] = lane_end[best];
    lane_end[best] += est[e].nrounds;
  }
  int64_t nglobal = 0;
  for (int64_t v : lane_end) nglobal = std::max(nglobal, v);
  std::vector<int64_t> seg_start;
  std::vector<int2> seg;
  {
    // estimations active in each global round, in estimation order
    std::vector<std::vector<int>> begin_at(nglobal + 1);
    for (int e = 0; e < count; ++e) begin_at[start[e]].push_back(e);
    std::vector<int> active;
    int64_t cum = 0;
    for (int64_t Rg = 0; Rg < nglobal; ++Rg) {
      if (!begin_at[Rg].empty()) {
        active.insert(active.end(), begin_at[Rg].begin(), begin_at[Rg].end());
        std::sort(active.begin(), active.end());
      }
      size_t keep = 0;
      for (size_t q = 0; q < active.size(); ++q) {
        const int e = active[q];
        const int64_t k = Rg - start[e];
        const int64_t n = rs[e][k + 1] - rs[e][k];
        if (n > 0) {
          seg_start.push_back(cum);
          seg.push_back(make_int2(e, (int)k));
          cum += n;
        }
        if (k + 1 < est[e].nrounds) active[keep++] = e;
      }
      active.resize(keep);
    }
    seg_start.push_back(cum);
  }
  const int64_t nseg = (int64_t)seg.size();
  const int64_t total = seg_start.back();

  // device arena: [staged: descriptors | FFT plans | seg_start | seg | per estimation:
  // scalars, round starts] [counters: per estimation cnt, fin | next, error] [per
  // estimation: ring slots, Welford state]
  size_t staged = 0;
  const size_t off_est = staged;
  staged = align256(staged + sizeof(EngineEst) * count);
  const size_t off_plan = staged;
  staged = align256(staged + sizeof(FftPlan) * 4 * count);
  const size_t off_segs = staged;
  staged = align256(staged + sizeof(int64_t) * (nseg + 1));
  const size_t off_seg = staged;
  staged = align256(staged + sizeof(int2) * std::max<int64_t>(nseg, 1));
  std::vector<size_t> off_sc(count), off_rs(count), off_cnt(count), off_slot(count);
  for (int e = 0; e < count; ++e) {
    off_sc[e] = staged;
    staged = align256(staged + sizeof(double) * 3 * est[e].S);
    off_rs[e] = staged;
    staged = align256(staged + sizeof(int64_t) * rs[e].size());
  }
  size_t counters = staged;
  for (int e = 0; e < count; ++e) {
    off_cnt[e] = counters;
    counters = align256(counters + sizeof(int) * ((size_t)est[e].NB * est[e].P + (size_t)est[e].NB * est[e].Tf));
  }
  const size_t off_flags = counters;
  counters = align256(counters + 2 * sizeof(int));
  size_t total_bytes = counters;
  for (int e = 0; e < count; ++e) {
    off_slot[e] = total_bytes;
    total_bytes = align256(total_bytes + sizeof(double2) * (size_t)est[e].Q * est[e].slot_elems +
                           sizeof(double) * 4 * (size_t)est[e].G);
  }
  char *m = (char *)ensure(ctx, BUF_ENGINE, total_bytes);
  std::vector<char> host(staged, 0);
  for (int e = 0; e < count; ++e) {
    EngineEst &E = est[e];
    double *sc = (double *)(m + off_sc[e]);
    E.cw = sc;
    E.vscale = sc + E.S;
    E.dlogt = sc + 2 * E.S;
    E.round_start = (const int64_t *)(m + off_rs[e]);
    E.cnt = (int *)(m + off_cnt[e]);
    E.fin = E.cnt + E.NB * E.P;
    E.slots = (double2 *)(m + off_slot[e]);
    E.plan = (const FftPlan *)(m + off_plan) + 4 * e;
    std::memcpy(host.data() + off_plan + sizeof(FftPlan) * 4 * e, plans[e].data(), sizeof(FftPlan) * 4);
    E.wstate = (double *)(m + off_slot[e] + sizeof(double2) * (size_t)E.Q * E.slot_elems);
    double *hsc = (double *)(host.data() + off_sc[e]);
    std::memcpy(hsc, args[e].cw, sizeof(double) * E.S);
    std::memcpy(hsc + E.S, args[e].vscale, sizeof(double) * E.S);
    std::memcpy(hsc + 2 * E.S, args[e].dlogt, sizeof(double) * E.S);
    std::memcpy(host.data() + off_rs[e], rs[e].data(), sizeof(int64_t) * rs[e].size());
  }
  std::memcpy(host.data() + off_est, est.data(), sizeof(EngineEst) * count);
  std::memcpy(host.data() + off_segs, seg_start.data(), sizeof(int64_t) * (nseg + 1));
  if (nseg) std::memcpy(host.data() + off_seg, seg.data(), sizeof(int2) * nseg);
  PKDE_CUDA_TRY(cudaMemcpyAsync(m, host.data(), staged, cudaMemcpyHostToDevice, st));
  PKDE_CUDA_TRY(cudaMemsetAsync(m + staged, 0, counters - staged, st));
  R.est = (const EngineEst *)(m + off_est);
  R.count = count;
  R.seg_start = (const int64_t *)(m + off_segs);
  R.seg = (const int2 *)(m + off_seg);
  R.nseg = nseg;
  R.total_items = total;
  R.next = (int *)(m + off_flags);
  R.error = R.next + 1;
  R.spin_limit = (long long)ctx->wait_limit;
  bool any_gen = false;
  for (int e = 0; e < count; ++e)
    for (int j = 0; j < est[e].ndim; ++j) any_gen |= est[e].gen[j] != 0;
  auto kern = any_gen ? engine_kernel<true> : engine_kernel<false>;
  // the state region doubles as the second exchange buffer of the register-FFT axis passes
  const size_t state_elems = std::max<size_t>(max_reg_tile, 8 * kEngineThreads);
  const size_t smem = sizeof(double2) * (max_tile + state_elems + max_tw);
  allow_dynamic_smem(ctx, kern, smem);
  int per_sm = 0;
  PKDE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kEngineThreads, smem));
  if (per_sm < 1) throw Error{PKDE_EUNSUPPORTED, "engine kernel does not fit on an SM"};
  const int64_t grid = std::min<int64_t>(total, (int64_t)per_sm * ctx->sm_count);
  if (grid > 0) {
    Trace tr(ctx, PKDE_PHASE_STEP_VMR, st);
    kern<<<(unsigned)grid, kEngineThreads, smem, st>>>(R, (int)max_tile, (int)state_elems);
  }
  PKDE_CHECK_LAUNCH();
  // the launch's error flag comes back with the call's own synchronisation
  constexpr int kEngineFlags = 64;
  if (!ctx->engine_flags) PKDE_CUDA_TRY(cudaMallocHost(&ctx->engine_flags, sizeof(int) * kEngineFlags));
  if (ctx->engine_flags_used == kEngineFlags) {  // every slot in use: check them first
    PKDE_CUDA_TRY(cudaStreamSynchronize(st));
    check_engine_flags(ctx);
  }
  int *flag = ctx->engine_flags + ctx->engine_flags_used++;
  PKDE_CUDA_TRY(cudaMemcpyAsync(flag, R.error, sizeof(int), cudaMemcpyDeviceToHost, st));
}

void check_engine_flags(pkde_ctx *ctx) {
  bool bad = false;
  for (int i = 0; i < ctx->engine_flags_used; ++i) bad |= ctx->engine_flags[i] != 0;
  ctx->engine_flags_used = 0;
  if (bad) throw Error{PKDE_ECUDA, "step engine: a dependency wait timed out (run aborted)"};
}

void run_engine(pkde_ctx *ctx, const EngineArgs &A, cudaStream_t st) { run_engine_batch(ctx, &A, 1, st); }

size_t engine_ring_bytes(const EngineArgs &A) {
  const EngineEst E = describe(A);
  return sizeof(double2) * (size_t)E.Q * (size_t)E.slot_elems;
}

// ---------------------------------------------------------------- autotuning
// Key of a shape: grid dimensions and pairs of bootstraps (the schedule depends on
// nothing else).
static std::string tune_key(const EngineArgs &A) {
  std::string k = std::to_string(A.grid->ndim);
  for (int j = 0; j < A.grid->ndim; ++j) k += "x" + std::to_string(A.grid->dims[j]);
  return k + ":p" + std::to_string(A.npairs);
}

static void load_tune_file(pkde_ctx *ctx) {
  if (ctx->tune_loaded) return;
  ctx->tune_loaded = true;
  const char *path = getenv("PKDE_TUNE_CACHE");
  if (!path || !*path) return;
  FILE *f = fopen(path, "r");
  if (!f) return;
  char key[256];
  int a, b, c;
  while (fscanf(f, "%255s %d %d %d", key, &a, &b, &c) == 4) ctx->tune[key] = {a, b, c};
  fclose(f);
}

static void save_tune(pkde_ctx *ctx, const std::string &key, const std::array<int, 3> &v) {
  const char *path = getenv("PKDE_TUNE_CACHE");
  if (!path || !*path) return;
  FILE *f = fopen(path, "a");
  if (!f) return;
  fprintf(f, "%s %d %d %d\n", key.c_str(), v[0], v[1], v[2]);
  fclose(f);
}

void autotune_engine(pkde_ctx *ctx, EngineArgs &A, cudaStream_t st) {
  load_tune_file(ctx);
  const std::string key = tune_key(A);
  auto it = ctx->tune.find(key);
  if (it == ctx->tune.end()) {
    if (!ctx->autotune) return;
    // trial runs over the first bandwidth steps of this estimation
    EngineArgs T = A;
    T.S = std::min(A.S, 16);
    const bool twoD = A.grid->ndim == 2;
    std::vector<std::array<int, 3>> cand;
    for (int slot : {8, 16, 32, 64})
      for (int tpi : {1, 2, 4, 8}) cand.push_back({slot, tpi, 2});
    // Wide groups: ring slots holding half or all of the bootstrap pairs.  With all pairs in
    // one group a step has a single pair batch, so the final pass reads and writes the
    // per-point Welford state once per step and no group waits for the previous one
    // (measured: 512 x 512 / B = 64 engine 57.1 -> 53.2 ms, 128^3 / B = 32 252 -> 207 ms).
    // Only where the slot exceeds the narrow sizes above and the ring (at the largest delay
    // tried) stays within an eighth of the free device memory.
    size_t freeb = 0, totalb = 0;
    PKDE_CUDA_TRY(cudaMemGetInfo(&freeb, &totalb));
    const size_t budget = freeb / 8;
    auto ring_fits = [&](const std::array<int, 3> &c) {
      EngineArgs R = A;
      R.tune_slot_mb = c[0];
      R.tune_tpi = c[1];
      R.tune_delay = c[2];
      return engine_ring_bytes(R) <= budget;
    };
    if (ctx->tune_wide) {
      const int64_t pair_bytes = (int64_t)sizeof(double2) * 2 * grid_size(A.grid);
      int last_mb = 0;
      for (int gg : {(A.npairs + 1) / 2, A.npairs}) {
        const int64_t mb = (gg * pair_bytes + (1 << 20) - 1) >> 20;
        if (mb <= kNarrowSlotMB || mb == last_mb || mb > (1 << 30)) continue;
        last_mb = (int)mb;
        for (int tpi : {2, 4, 8})
          if (ring_fits({(int)mb, tpi, 4})) cand.push_back({(int)mb, tpi, 2});
      }
    }
    cudaEvent_t e0, e1;
    PKDE_CUDA_TRY(cudaEventCreate(&e0));
    PKDE_CUDA_TRY(cudaEventCreate(&e1));
    auto trial = [&](const std::array<int, 3> &c) {
      T.tune_slot_mb = c[0];
      T.tune_tpi = c[1];
      T.tune_delay = c[2];
      run_engine_batch(ctx, &T, 1, st);  // warm (buffers sized, code loaded)
      PKDE_CUDA_TRY(cudaEventRecord(e0, st));
      run_engine_batch(ctx, &T, 1, st);
      PKDE_CUDA_TRY(cudaEventRecord(e1, st));
      PKDE_CUDA_TRY(cudaEventSynchronize(e1));
      check_engine_flags(ctx);
      float ms = 0.f;
      PKDE_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
      return ms;
    };
    std::array<int, 3> best = {32, twoD ? 2 : 8, 2};
    float best_ms = trial(best);
    for (const auto &c : cand) {
      const float ms = trial(c);
      if (ms < best_ms) best_ms = ms, best = c;
    }
    for (int d : {3, 4}) {
      std::array<int, 3> c = best;
      c[2] = d;
      const float ms = trial(c);
      if (ms < best_ms) best_ms = ms, best = c;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    it = ctx->tune.emplace(key, best).first;
    save_tune(ctx, key, best);
  }
  A.tune_slot_mb = it->second[0];
  A.tune_tpi = it->second[1];
  A.tune_delay = it->second[2];
}

}  // namespace pkde
