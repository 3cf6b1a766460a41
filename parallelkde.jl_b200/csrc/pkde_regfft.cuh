// Register-resident FP64 FFT of a tile of power-of-two lines (N = 2^LOGN, 16..4096).
//
// Each thread owns one radix-8 butterfly of one line: 8 complex values in registers.
// The first stage takes its inputs straight from the caller (global memory), the last
// stage leaves its outputs in registers, and the stages in between exchange through
// a padded shared-memory tile.  Stages are Stockham radix 8, then one radix-4 or
// radix-2 stage for the remaining factor.
//
// Thread-to-work mapping (compile-time choice):
//   ROWS: consecutive lanes take consecutive butterflies of one line -- global access
//         along a contiguous line (grid axis 1) is coalesced;
//   COLS: consecutive lanes take the same butterfly of consecutive lines -- global
//         access across adjacent lines (any other axis) is coalesced.
// Shared-memory layout: line l at l*LP, element i at pad8(i) = i + i/8; LP is chosen so
// that in both mappings every quarter-warp of 16-byte accesses hits 8 distinct bank
// groups.  Twiddles come from per-stage tables laid out [r][k] (k fastest).
#pragma once

#include "pkde_internal.cuh"

namespace pkde {

__host__ __device__ constexpr int pad8(int i) { return i + (i >> 3); }
__host__ __device__ constexpr int cilog2(int v) { return v <= 1 ? 0 : 1 + cilog2(v >> 1); }

// Tile geometry for lines of N = 2^LOGN points; NLINES lines per tile (default: enough
// lines for at least 256 threads).
template <int LOGN, int NLINES = 0>
struct Pow2 {
  static constexpr int N = 1 << LOGN;
  static constexpr int NB8 = N / 8;                       // butterflies per line per radix-8 stage
  static constexpr int NST8 = LOGN / 3;                   // radix-8 stages
  static constexpr int REM = LOGN % 3;                    // 1: radix-2 tail, 2: radix-4 tail
  static constexpr int NL = NLINES > 0 ? NLINES : (NB8 > 256 ? 1 : 256 / NB8);  // lines per tile
  static constexpr int THREADS = NL * NB8;                // one butterfly per thread
  static constexpr int LPAD = pad8(N);                    // padded line length before skew
  // skew so that NL lines interleave over the 8 bank groups in COLS mode
  static constexpr int SKEW = NL >= 8 ? 1 : 8 / NL;
  static constexpr int LP = LPAD + ((SKEW - (LPAD % 8)) % 8 + 8) % 8;
  static constexpr int TILE = NL * LP;                    // complex values in the tile
  // twiddle tables: stage ST >= 1 of radix 8 has 7 * 8^ST entries, the tail 3*N/4 or N/2
  __host__ __device__ static constexpr int tw_stage_off(int st) {
    int off = 0, ns = 8;
    for (int s = 1; s < st; ++s, ns *= 8) off += 7 * ns;
    return off;
  }
  static constexpr int TW8 = tw_stage_off(NST8);          // entries of all radix-8 tables
  static constexpr int TWTAIL = REM == 2 ? 3 * (N / 4) : (REM == 1 ? N / 2 : 0);
  static constexpr int TWSIZE = TW8 + TWTAIL;
};

// Host: per-stage twiddle tables (cos, sin)(2 pi m / N) in the order used on the device.
inline std::vector<double2> make_stage_twiddles(int logn) {
  const int N = 1 << logn;
  const int nst8 = logn / 3, rem = logn % 3;
  std::vector<double2> out;
  const long double two_pi = 6.283185307179586476925286766559005768L;
  auto w = [&](long long m) {
    long double a = two_pi * (long double)(m % N) / (long double)N;
    return make_double2((double)cosl(a), (double)sinl(a));
  };
  for (int st = 1, ns = 8; st < nst8; ++st, ns *= 8) {
    const int tshift = logn - 3 * st - 3;
    for (int r = 1; r < 8; ++r)
      for (int k = 0; k < ns; ++k) out.push_back(w((long long)(r * k) << tshift));
  }
  const int ns_tail = 1 << (3 * nst8);
  if (rem == 2)
    for (int r = 1; r < 4; ++r)
      for (int k = 0; k < ns_tail; ++k) out.push_back(w((long long)r * k));
  if (rem == 1)
    for (int k = 0; k < ns_tail; ++k) out.push_back(w(k));
  return out;
}

// Synchronisation of the threads that share one line.  In ROWS mapping a line belongs
// to NB8 consecutive threads: whole warps (named barrier 1 + line, NB8 threads) or a
// part of one warp (__syncwarp).  In COLS mapping lines interleave across the block,
// so the whole block synchronises.
template <int LOGN, bool COLS, int NLINES>
__device__ __forceinline__ void line_sync(int line) {
  constexpr int NB8 = Pow2<LOGN, NLINES>::NB8;
  if constexpr (COLS) {
    __syncthreads();
  } else if constexpr (NB8 >= 32) {
    if constexpr (Pow2<LOGN, NLINES>::NL == 1) {
      __syncthreads();
    } else {
      asm volatile("bar.sync %0, %1;" ::"r"(1 + line), "r"(NB8) : "memory");
    }
  } else {
    __syncwarp();
  }
}

template <int DIR>
__device__ __forceinline__ double2 twr(const double2 *tw, int i) {
  const double2 w = tw[i];
  return make_double2(w.x, DIR > 0 ? w.y : -w.y);
}

template <int LOGN, bool COLS, int NLINES = 0>
struct TileIdx {
  using P = Pow2<LOGN, NLINES>;
  __device__ __forceinline__ static int line() {
    return COLS ? (threadIdx.x & (P::NL - 1)) : (threadIdx.x >> (LOGN - 3));
  }
  __device__ __forceinline__ static int bfly() {
    return COLS ? (threadIdx.x >> cilog2(P::NL)) : (threadIdx.x & (P::NB8 - 1));
  }
};

// Position (within the line) of output value i of the last stage for butterfly t.
template <int LOGN>
__device__ __forceinline__ int out_pos(int t, int i) {
  using P = Pow2<LOGN>;
  if constexpr (P::REM == 0) return t + i * P::NB8;
  if constexpr (P::REM == 2) return t + (i >> 2) * P::NB8 + (i & 3) * (P::N / 4);
  return t + (i >> 1) * P::NB8 + (i & 1) * (P::N / 2);
}
// Position of input value r of the first stage for butterfly t (radix 8 first stage).
template <int LOGN>
__device__ __forceinline__ int in_pos(int t, int r) {
  return t + r * Pow2<LOGN>::NB8;
}

// Radix-8 stage ST on v (inputs of butterfly t); outputs written to the tile line.
template <int LOGN, int DIR, int ST>
__device__ __forceinline__ void stage8_compute(double2 *v, int t, const double2 *tw) {
  constexpr int LNS = 3 * ST;
  constexpr int NS = 1 << LNS;
  if constexpr (ST > 0) {
    const int k = t & (NS - 1);
    const double2 *tws = tw + Pow2<LOGN>::tw_stage_off(ST);
#pragma unroll
    for (int r = 1; r < 8; ++r) v[r] = cmul(v[r], twr<DIR>(tws, (r - 1) * NS + k));
  }
  dft8<DIR>(v);
}

template <int LOGN, int ST>
__device__ __forceinline__ void stage8_store(double2 *line, const double2 *v, int t) {
  constexpr int LNS = 3 * ST;
  constexpr int NS = 1 << LNS;
  const int d = ((t >> LNS) << (LNS + 3)) + (t & (NS - 1));
#pragma unroll
  for (int q = 0; q < 8; ++q) line[pad8(d + q * NS)] = v[q];
}

template <int LOGN>
__device__ __forceinline__ void load8(const double2 *line, double2 *v, int t) {
#pragma unroll
  for (int r = 0; r < 8; ++r) v[r] = line[pad8(t + r * Pow2<LOGN>::NB8)];
}

// Tail stages: the thread's two radix-4 (or four radix-2) butterflies.
template <int LOGN, int DIR>
__device__ __forceinline__ void tail4(double2 *line, double2 *v, int t, const double2 *tw) {
  using P = Pow2<LOGN>;
  constexpr int NS = 1 << (3 * P::NST8);
  constexpr int NB4 = P::N / 4;
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int r = 0; r < 4; ++r) v[h * 4 + r] = line[pad8(t + h * P::NB8 + r * NB4)];
  const double2 *tws = tw + P::TW8;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int k = (t + h * P::NB8) & (NS - 1);
#pragma unroll
    for (int r = 1; r < 4; ++r) v[h * 4 + r] = cmul(v[h * 4 + r], twr<DIR>(tws, (r - 1) * NS + k));
    dft4<DIR>(v + h * 4);
  }
}

template <int LOGN, int DIR>
__device__ __forceinline__ void tail2(double2 *line, double2 *v, int t, const double2 *tw) {
  using P = Pow2<LOGN>;
  constexpr int NS = 1 << (3 * P::NST8);
  constexpr int NB2 = P::N / 2;
#pragma unroll
  for (int h = 0; h < 4; ++h)
#pragma unroll
    for (int r = 0; r < 2; ++r) v[h * 2 + r] = line[pad8(t + h * P::NB8 + r * NB2)];
  const double2 *tws = tw + P::TW8;
#pragma unroll
  for (int h = 0; h < 4; ++h) {
    const int k = (t + h * P::NB8) & (NS - 1);
    v[h * 2 + 1] = cmul(v[h * 2 + 1], twr<DIR>(tws, k));
    dft2<DIR>(v + h * 2);
  }
}

// DB (double buffering): exchange k (the store of stage k) goes to buffer k % 2, so the
// barrier after each load is not needed: the next store goes to the other buffer, and
// the store after that follows another barrier that every thread reaches only after its
// loads.  The tile is free for the next call when the last exchange used buffer 1; after
// an exchange through buffer 0 a trailing barrier keeps that guarantee.
template <int LOGN, int DIR, int ST, bool COLS, int NLINES, bool DB = false>
__device__ __forceinline__ void run_stages(double2 *line, double2 *line2, double2 *v, int t, const double2 *tw,
                                           int l) {
  using P = Pow2<LOGN>;
  stage8_compute<LOGN, DIR, ST>(v, t, tw);
  constexpr bool last8 = ST + 1 == P::NST8;
  double2 *buf = (DB && (ST & 1)) ? line2 : line;
  if constexpr (last8 && P::REM == 0) {
    if constexpr (DB && ST >= 1 && ((ST - 1) & 1) == 0) line_sync<LOGN, COLS, NLINES>(l);
    return;  // outputs stay in registers: v[q] = X[t + q*N/8]
  } else {
    stage8_store<LOGN, ST>(buf, v, t);
    line_sync<LOGN, COLS, NLINES>(l);
    if constexpr (!last8) {
      load8<LOGN>(buf, v, t);
      if constexpr (!DB) line_sync<LOGN, COLS, NLINES>(l);
      run_stages<LOGN, DIR, ST + 1, COLS, NLINES, DB>(line, line2, v, t, tw, l);
    } else if constexpr (P::REM == 2) {
      tail4<LOGN, DIR>(buf, v, t, tw);
      if constexpr (!DB || (ST & 1) == 0) line_sync<LOGN, COLS, NLINES>(l);
    } else {
      tail2<LOGN, DIR>(buf, v, t, tw);
      if constexpr (!DB || (ST & 1) == 0) line_sync<LOGN, COLS, NLINES>(l);
    }
  }
}

// FFT of the thread's line.  On entry v[r] = x[in_pos(t, r)]; on exit v[i] =
// X[out_pos(t, i)].  Every thread of the line (COLS: of the block) must call it; the
// line's tile memory (and tile2 with DB) is free again for the next call when it returns.
template <int LOGN, int DIR, bool COLS, int NLINES = 0, bool DB = false>
__device__ __forceinline__ void tile_fft_reg(double2 *tile, double2 *v, const double2 *tw, double2 *tile2 = nullptr) {
  using P = Pow2<LOGN, NLINES>;
  using I = TileIdx<LOGN, COLS, NLINES>;
  const int l = I::line();
  run_stages<LOGN, DIR, 0, COLS, NLINES, DB>(tile + l * P::LP, DB ? tile2 + l * P::LP : nullptr, v, I::bfly(), tw,
                                             l);
}

}  // namespace pkde
