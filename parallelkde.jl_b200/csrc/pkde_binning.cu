// Dirac-sequence binning (cloud-in-cell of every bootstrap resample onto the grid).
//
// Reference: src/StatisticsPropagation/DirectSpace.jl:196-242 (generate_dirac_cpu!, the
// FP64 arithmetic followed here), :364-477 (generate_dirac_cuda!, FP32 atomics),
// :479-512 (check_data).
//
// B200 design: the per-sample arithmetic (cell index, remainders, the 2^N corner terms)
// is done once per sample in FP64 exactly as the reference's CPU path does it; each
// term is then quantised to a 64-bit fixed-point integer with a power-of-two scale
// chosen from the exact per-cell draw counts, so that the per-cell sums are exact
// integer sums: independent of the order in which the atomics land, and within one
// rounding of the term values.  Draws are processed bootstrap-major so the atomics of
// one bootstrap column stay in L2.
#include <cstring>
#include <mutex>

#include "pkde_internal.cuh"

namespace pkde {
namespace {

constexpr int kThreads = 256;

struct GridDev {
  int ndim;
  int64_t dims[4];
  int64_t stride[4];
  double lo[4], hi[4], h[4];
};

GridDev to_dev(const pkde_grid *g) {
  GridDev d{};
  d.ndim = g->ndim;
  int64_t s = 1;
  for (int j = 0; j < g->ndim; ++j) {
    d.dims[j] = g->dims[j];
    d.stride[j] = s;
    s *= g->dims[j];
    d.lo[j] = g->lo[j];
    d.hi[j] = g->hi[j];
    d.h[j] = g->h[j];
  }
  return d;
}

// Per sample: bounds check, lower cell, remainders r_h (DirectSpace.jl:219-224).
__global__ void prepass_kernel(GridDev g, const double *__restrict__ data, int64_t n,
                               uint32_t *__restrict__ cell, double *__restrict__ rh, int *err) {
  int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= n) return;
  int64_t c = 0;
  bool bad_bound = false, bad_top = false;
  for (int j = 0; j < g.ndim; ++j) {
    double x = data[s * g.ndim + j];
    if ((x >= g.hi[j]) | (x <= g.lo[j]) | !(x == x)) bad_bound = true;
    double delta = __dsub_rn(x, g.lo[j]);
    double l = floor(__ddiv_rn(delta, g.h[j]));
    double r = fmod(delta, g.h[j]);
    if (!bad_bound && (l + 1.0 >= (double)g.dims[j] || l < 0.0)) bad_top = true;
    int64_t li = bad_bound || bad_top ? 0 : (int64_t)l;
    c += li * g.stride[j];
    rh[j * n + s] = r;
  }
  if (bad_bound) atomicOr(err, 1);
  if (bad_top) atomicOr(err, 2);
  cell[s] = (uint32_t)c;
}

__device__ __forceinline__ int64_t draw_sample(int64_t b, int64_t j, int64_t n, int64_t nboot,
                                               const int32_t *__restrict__ idx, uint64_t seed, int *err) {
  if (b == nboot) return j;  // identity resample (B = 0 in the reference)
  if (idx) {
    int64_t v = (int64_t)idx[b * n + j] - 1;
    if (v < 0 || v >= n) {
      atomicOr(err, 4);
      return 0;
    }
    return v;
  }
  return boot_draw(seed, n, b, j);
}

// counts[b][cell]: draws of resample b whose lower cell is `cell` (slot nboot = identity).
__global__ void count_kernel(const uint32_t *__restrict__ cell, int64_t n, int64_t nslots, int64_t nboot,
                             int64_t G, const int32_t *__restrict__ idx, uint64_t seed,
                             uint32_t *__restrict__ counts, int *err) {
  const int64_t total = nslots * n;
  for (int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; d < total;
       d += (int64_t)gridDim.x * blockDim.x) {
    int64_t b = d / n;
    int64_t j = d - b * n;
    int64_t slot_b = b < nboot ? b : nboot;  // slots beyond nboot only exist for identity
    int64_t s = draw_sample(slot_b, j, n, nboot, idx, seed, err);
    atomicAdd(&counts[b * G + cell[s]], 1u);
  }
}

__global__ void max_kernel(const uint32_t *__restrict__ v, int64_t m, unsigned int *out) {
  uint32_t best = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
    best = max(best, v[i]);
  for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, best);
}

// Per sample: the 2^N corner terms of DirectSpace.jl:227-237, quantised.
// Corner c: axis j (0-based) takes the lower cell iff bit (N-1-j) of c is set.
__global__ void quantize_kernel(GridDev g, const double *__restrict__ rh, int64_t n, double denom,
                                int e_m, int e_v, unsigned long long *__restrict__ qm,
                                unsigned long long *__restrict__ qv) {
  int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int N = g.ndim;
  double r_h[4], r_l[4];
  for (int j = 0; j < N; ++j) {
    r_h[j] = rh[j * n + s];
    r_l[j] = __dsub_rn(g.h[j], r_h[j]);
  }
  const int nc = 1 << N;
  for (int c = 0; c < nc; ++c) {
    double pl = 1.0, ph = 1.0;
    bool fl = false, fh = false;
    for (int j = 0; j < N; ++j) {
      if ((c >> (N - 1 - j)) & 1) {
        pl = fl ? __dmul_rn(pl, r_l[j]) : r_l[j];
        fl = true;
      } else {
        ph = fh ? __dmul_rn(ph, r_h[j]) : r_h[j];
        fh = true;
      }
    }
    double term = __ddiv_rn(__dmul_rn(pl, ph), denom);
    double sq = __dmul_rn(term, term);
    qm[c * n + s] = __double2ull_rn(ldexp(term, e_m));
    if (qv) qv[c * n + s] = __double2ull_rn(ldexp(sq, e_v));
  }
}

// Scatter of the quantised terms.  Destination u64 slot of (resample b, cell, array):
//   paired layout (spectra): ((2*(b/2) + arr) * G + cell) * 2 + (b % 2), identity slot
//   (b == nboot) at (2*npairs*G + cell) * 2;  plain layout: arr_base[arr] + b*G + cell.
template <bool PAIRED>
__global__ void weight_kernel(const uint32_t *__restrict__ cell, int64_t n, int64_t nslots, int64_t nboot,
                              int64_t G, int ndim, const int64_t *__restrict__ corner_off,
                              const int32_t *__restrict__ idx, uint64_t seed,
                              const unsigned long long *__restrict__ qm,
                              const unsigned long long *__restrict__ qv, unsigned long long *__restrict__ outM,
                              unsigned long long *__restrict__ outV, int64_t npairs, int *err) {
  const int64_t total = nslots * n;
  const int nc = 1 << ndim;
  for (int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; d < total;
       d += (int64_t)gridDim.x * blockDim.x) {
    int64_t b = d / n;
    int64_t j = d - b * n;
    int64_t s = draw_sample(b < nboot ? b : nboot, j, n, nboot, idx, seed, err);
    int64_t c0 = cell[s];
    for (int c = 0; c < nc; ++c) {
      int64_t cc = c0 + corner_off[c];
      unsigned long long m = qm[c * n + s];
      if (PAIRED) {
        if (b == nboot) {
          atomicAdd(&outM[(2 * npairs * G + cc) * 2], m);
        } else {
          int64_t p = b >> 1, lane = b & 1;
          atomicAdd(&outM[((2 * p) * G + cc) * 2 + lane], m);
          if (qv) atomicAdd(&outM[((2 * p + 1) * G + cc) * 2 + lane], qv[c * n + s]);
        }
      } else {
        atomicAdd(&outM[b * G + cc], m);
        if (qv && outV && b < nboot) atomicAdd(&outV[b * G + cc], qv[c * n + s]);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Estimator scatter in cell order.  The samples are sorted by lower cell once (a counting
// sort from the identity counts); each bootstrap's draws become per-sample
// multiplicities m[b][i] (i = position in cell order); the scatter then walks (b, i) in
// order and adds m * term.  Neighbouring threads hit neighbouring cells, and within a
// warp the contributions of equal cells are summed (segmented scan) before one atomic.
// All sums are exact 64-bit integers, so the result equals the per-draw scatter's.

constexpr int kScanChunk = 2048;  // cells per block in the scans

// per-chunk sums of the identity counts (the samples per cell)
__global__ void cell_chunk_sum_kernel(const uint32_t *__restrict__ cnt, int64_t G, uint32_t *__restrict__ csum) {
  __shared__ uint32_t sh[kThreads / 32];
  const int64_t c0 = (int64_t)blockIdx.x * kScanChunk;
  uint32_t v = 0;
  for (int k = threadIdx.x; k < kScanChunk; k += blockDim.x)
    if (c0 + k < G) v += cnt[c0 + k];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < kThreads / 32; ++w) t += sh[w];
    csum[blockIdx.x] = t;
  }
}

// exclusive scan of the chunk sums (one block, in order)
__global__ void chunk_scan_kernel(uint32_t *csum, int64_t nchunks) {
  if (threadIdx.x != 0) return;
  uint32_t run = 0;
  for (int64_t k = 0; k < nchunks; ++k) {
    const uint32_t v = csum[k];
    csum[k] = run;
    run += v;
  }
}

// cstart[c] = first position of cell c in cell order (exclusive scan of the counts);
// also clears the per-cell fill counters
__global__ void cell_start_kernel(const uint32_t *__restrict__ cnt, int64_t G, const uint32_t *__restrict__ csum,
                                  uint32_t *__restrict__ cstart, uint32_t *__restrict__ cfill) {
  __shared__ uint32_t part[kThreads];
  const int64_t c0 = (int64_t)blockIdx.x * kScanChunk;
  constexpr int PER = kScanChunk / kThreads;
  uint32_t v[PER];
  uint32_t t = 0;
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int64_t c = c0 + threadIdx.x * PER + q;
    v[q] = c < G ? cnt[c] : 0u;
    t += v[q];
  }
  part[threadIdx.x] = t;
  __syncthreads();
  if (threadIdx.x == 0) {  // exclusive scan of the per-thread sums (256 values)
    uint32_t run = csum[blockIdx.x];
    for (int k = 0; k < kThreads; ++k) {
      const uint32_t x = part[k];
      part[k] = run;
      run += x;
    }
  }
  __syncthreads();
  uint32_t run = part[threadIdx.x];
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int64_t c = c0 + threadIdx.x * PER + q;
    if (c < G) {
      cstart[c] = run;
      cfill[c] = 0u;
    }
    run += v[q];
  }
}

// pos[s] = position of sample s in cell order; cell_sorted[pos] = its lower cell
__global__ void cell_sort_kernel(const uint32_t *__restrict__ cell, int64_t n, const uint32_t *__restrict__ cstart,
                                 uint32_t *__restrict__ cfill, uint32_t *__restrict__ pos,
                                 uint32_t *__restrict__ cell_sorted) {
  for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t c = cell[s];
    const uint32_t p = cstart[c] + atomicAdd(&cfill[c], 1u);
    pos[s] = p;
    cell_sorted[p] = c;
  }
}

// mult[b * n + pos[s]] = how often resample b draws sample s
__global__ void mult_kernel(int64_t n, int64_t nboot, const int32_t *__restrict__ idx, uint64_t seed,
                            const uint32_t *__restrict__ pos, uint32_t *__restrict__ mult, int *err) {
  const int64_t total = nboot * n;
  for (int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; d < total; d += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = d / n;
    const int64_t j = d - b * n;
    const int64_t s = draw_sample(b, j, n, nboot, idx, seed, err);
    atomicAdd(&mult[b * n + pos[s]], 1u);
  }
}

// counts[b][cell] for the bootstrap resamples, summed from the multiplicities in cell
// order instead of one atomic per draw: the lanes of a warp hold consecutive (resample,
// position) entries, a segmented shuffle scan sums equal (resample, cell) keys, and the
// last lane of each run adds the run's sum with one atomic.
__global__ void resample_count_kernel(const uint32_t *__restrict__ cell_sorted, int64_t n, int64_t nboot, int64_t G,
                                      const uint32_t *__restrict__ mult, uint32_t *__restrict__ counts) {
  const int lane = threadIdx.x & 31;
  const int64_t total = nboot * n;
  // the loop bound is rounded up to whole warps, so the shuffles always see all 32 lanes
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; d - lane < total; d += stride) {
    const bool act = d < total;
    const int64_t b = act ? d / n : 0;
    const int64_t i = act ? d - b * n : 0;
    uint32_t v = act ? mult[d] : 0u;
    const uint32_t c0 = act ? cell_sorted[i] : 0u;
    const unsigned long long key = act ? (((unsigned long long)b << 32) | c0) : ~0ull - (unsigned long long)lane;
    bool same[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      const unsigned long long up = __shfl_up_sync(0xffffffffu, key, 1 << k);
      same[k] = lane >= (1 << k) && up == key;
    }
    const bool last = __shfl_down_sync(0xffffffffu, key, 1) != key || lane == 31;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      const uint32_t u = __shfl_up_sync(0xffffffffu, v, 1 << k);
      if (same[k]) v += u;
    }
    if (act && last && v) atomicAdd(&counts[b * G + c0], v);
  }
}

// The quantised corner terms of DirectSpace.jl:227-237, stored at the sample's position
// in cell order (quantize_kernel's arithmetic).
__device__ __forceinline__ void quantize2(double v, int e, int L, unsigned long long &hi, long long &lo) {
  // v 2^e = hi + f (hi the nearest integer, |f| <= 1/2, both exact), lo = f 2^L rounded
  const double x = ldexp(v, e);
  const double xr = rint(x);
  hi = (unsigned long long)xr;
  lo = __double2ll_rn(ldexp(x - xr, L));
}

__global__ void quantize_sorted_kernel(GridDev g, const double *__restrict__ rh, int64_t n, double denom,
                                       const int *__restrict__ esc, const uint32_t *__restrict__ pos,
                                       unsigned long long *__restrict__ qm, unsigned long long *__restrict__ qv,
                                       long long *__restrict__ qm_lo, long long *__restrict__ qv_lo) {
  int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int e_m = esc[0], e_v = esc[1], L = esc[2];
  const int N = g.ndim;
  const int64_t ps = pos[s];
  double r_h[4], r_l[4];
  for (int j = 0; j < N; ++j) {
    r_h[j] = rh[j * n + s];
    r_l[j] = __dsub_rn(g.h[j], r_h[j]);
  }
  const int nc = 1 << N;
  for (int c = 0; c < nc; ++c) {
    double pl = 1.0, ph = 1.0;
    bool fl = false, fh = false;
    for (int j = 0; j < N; ++j) {
      if ((c >> (N - 1 - j)) & 1) {
        pl = fl ? __dmul_rn(pl, r_l[j]) : r_l[j];
        fl = true;
      } else {
        ph = fh ? __dmul_rn(ph, r_h[j]) : r_h[j];
        fh = true;
      }
    }
    double term = __ddiv_rn(__dmul_rn(pl, ph), denom);
    double sq = __dmul_rn(term, term);
    quantize2(term, e_m, L, qm[c * n + ps], qm_lo[c * n + ps]);
    quantize2(sq, e_v, L, qv[c * n + ps], qv_lo[c * n + ps]);
  }
}

// Scatter in cell order into the paired spectra slots.  Work item d = (chunk c, i),
// c-major: sample position i (cell order) for the BC resamples b = c BC .. c BC + BC - 1
// (b = nboot the identity, multiplicity 1).  The thread loads its sample's quantised
// corner terms once and reuses them for every resample of its chunk (the term arrays,
// 4 x 2^N x n words, need not stay in L2 across resamples).  Warp lanes hold consecutive
// items of one chunk, so in every iteration they share b and their keys (b, cell) are
// non-decreasing along the warp: equal keys are contiguous and an inclusive segmented
// scan sums each run; the run's last lane adds it with one atomic per part.
template <int N>
__global__ void weight_sorted_kernel(const uint32_t *__restrict__ cell_sorted, int64_t n, int64_t nboot, int64_t G,
                                     const int64_t *__restrict__ corner_off, const uint32_t *__restrict__ mult,
                                     const unsigned long long *__restrict__ qm,
                                     const unsigned long long *__restrict__ qv, const long long *__restrict__ qm_lo,
                                     const long long *__restrict__ qv_lo, unsigned long long *__restrict__ out,
                                     unsigned long long *__restrict__ out_lo, int64_t npairs, int BC, int64_t nchunk) {
  constexpr int nc = 1 << N;
  constexpr bool REG = N <= 3;  // terms held in registers (4-D: re-read, from L1)
  const int lane = threadIdx.x & 31;
  const int64_t total = nchunk * n;
  // every lane of a warp runs the same number of iterations (the loop bound is rounded
  // up to whole warps, the resample loop has the same trip count in every lane), so the
  // shuffles always see all 32 lanes
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; d - lane < total; d += stride) {
    const bool act = d < total;
    const int64_t c = act ? d / n : 0;
    const int64_t i = act ? d - c * n : 0;
    const uint32_t c0 = act ? cell_sorted[i] : 0u;
    const unsigned long long key = act ? (((unsigned long long)c << 32) | c0) : ~0ull - (unsigned long long)lane;
    bool same[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      const unsigned long long up = __shfl_up_sync(0xffffffffu, key, 1 << k);
      same[k] = lane >= (1 << k) && up == key;
    }
    const bool last = __shfl_down_sync(0xffffffffu, key, 1) != key || lane == 31;
    unsigned long long rqm[REG ? nc : 1], rqv[REG ? nc : 1];
    long long rlm[REG ? nc : 1], rlv[REG ? nc : 1];
    if constexpr (REG) {
#pragma unroll
      for (int q = 0; q < nc; ++q) {
        rqm[q] = act ? qm[q * n + i] : 0ull;
        rqv[q] = act ? qv[q * n + i] : 0ull;
        rlm[q] = act ? qm_lo[q * n + i] : 0ll;
        rlv[q] = act ? qv_lo[q * n + i] : 0ll;
      }
    }
    for (int bb = 0; bb < BC; ++bb) {
      const int64_t b = c * BC + bb;
      const bool ab = act && b <= nboot;
      const uint32_t m = ab ? (b == nboot ? 1u : mult[b * n + i]) : 0u;
      const int64_t p = b >> 1, half = b & 1;
#pragma unroll
      for (int q = 0; q < nc; ++q) {
        const int64_t cc = (int64_t)c0 + (act ? corner_off[q] : 0);
        const unsigned long long tm = REG ? rqm[q] : (m ? __ldg(qm + q * n + i) : 0ull);
        const unsigned long long tv = REG ? rqv[q] : (m ? __ldg(qv + q * n + i) : 0ull);
        const long long tlm = REG ? rlm[q] : (m ? __ldg(qm_lo + q * n + i) : 0ll);
        const long long tlv = REG ? rlv[q] : (m ? __ldg(qv_lo + q * n + i) : 0ll);
        unsigned long long vm = m ? (unsigned long long)m * tm : 0ull;
        unsigned long long vv = (m && b < nboot) ? (unsigned long long)m * tv : 0ull;
        // low parts: signed, summed modulo 2^64 (the true sums fit in 63 bits)
        unsigned long long lm = m ? (unsigned long long)((long long)m * tlm) : 0ull;
        unsigned long long lv = (m && b < nboot) ? (unsigned long long)((long long)m * tlv) : 0ull;
#pragma unroll
        for (int k = 0; k < 5; ++k) {
          const unsigned long long um = __shfl_up_sync(0xffffffffu, vm, 1 << k);
          const unsigned long long uv = __shfl_up_sync(0xffffffffu, vv, 1 << k);
          const unsigned long long ulm = __shfl_up_sync(0xffffffffu, lm, 1 << k);
          const unsigned long long ulv = __shfl_up_sync(0xffffffffu, lv, 1 << k);
          if (same[k]) {
            vm += um;
            vv += uv;
            lm += ulm;
            lv += ulv;
          }
        }
        if (ab && last) {
          if (b == nboot) {
            const int64_t o = (2 * npairs * G + cc) * 2;
            if (vm) atomicAdd(&out[o], vm);
            if (lm) atomicAdd(&out_lo[o], lm);
          } else {
            const int64_t om = ((2 * p) * G + cc) * 2 + half, ov = ((2 * p + 1) * G + cc) * 2 + half;
            if (vm) atomicAdd(&out[om], vm);
            if (vv) atomicAdd(&out[ov], vv);
            if (lm) atomicAdd(&out_lo[om], lm);
            if (lv) atomicAdd(&out_lo[ov], lv);
          }
        }
      }
    }
  }
}

// In-place conversion of the fixed-point sums to FP64 (same 8-byte slots).
__global__ void dequant_kernel(unsigned long long *v, int64_t m, double scale) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    unsigned long long x = v[i];
    reinterpret_cast<double *>(v)[i] = (double)x * scale;
  }
}

__global__ void dequant_paired_kernel(unsigned long long *v, int64_t G, int64_t npairs, double sm, double sv) {
  // arrays: [z0, w0, z1, w1, ..., zF]; w arrays use sv
  const int64_t total = (2 * npairs + 1) * G * 2;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t arr = i / (2 * G);
    double sc = (arr < 2 * npairs && (arr & 1)) ? sv : sm;
    unsigned long long x = v[i];
    reinterpret_cast<double *>(v)[i] = (double)x * sc;
  }
}

// The fixed-point exponents of a binning job from its largest count (misc[1]), on the
// device so that phase B needs no read-back: a cell sums at most 2^N * cmax terms, each
// <= tmax (means) or tmax^2 (second moments); e = 62 - the binary exponent of that bound.
// esc[0] = e_m, esc[1] = e_v.  The same operations, in the same order, as on the host.
__global__ void scale_exponents_kernel(const int *misc, double nc, double tmax, int *esc) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double cmax = (double)(uint32_t)misc[1];
  const double bm = __dmul_rn(__dmul_rn(nc, cmax > 1.0 ? cmax : 1.0), tmax);
  const double bv = __dmul_rn(bm, tmax);
  int ex_m, ex_v;
  frexp(bm, &ex_m);
  frexp(bv, &ex_v);
  esc[0] = 62 - ex_m;
  esc[1] = 62 - ex_v;
  // low parts (|lo| <= 2^(L-1) a term) of at most nc * cmax terms a cell stay below 2^62
  const unsigned long long terms = (unsigned long long)nc * (unsigned long long)(cmax > 1.0 ? cmax : 1.0);
  const int lg = terms <= 1 ? 0 : 64 - __clzll((long long)(terms - 1));
  esc[2] = 62 - lg;
}

// Conversion of the two-part fixed-point sums to FP64, in place: hi 2^-e + lo 2^-(e+L)
// with the exponents from device memory (w arrays use e_v).
__global__ void dequant_paired_esc_kernel(unsigned long long *v, const unsigned long long *lo, int64_t G,
                                          int64_t npairs, const int *esc) {
  const int L = esc[2];
  const double sm = ldexp(1.0, -esc[0]), sv = ldexp(1.0, -esc[1]);
  const int64_t total = (2 * npairs + 1) * G * 2;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t arr = i / (2 * G);
    double sc = (arr < 2 * npairs && (arr & 1)) ? sv : sm;
    const unsigned long long x = v[i];
    const double xl = (double)(long long)lo[i];
    reinterpret_cast<double *>(v)[i] = fma(ldexp(xl, -L), sc, (double)x * sc);
  }
}

int grid_blocks(pkde_ctx *ctx, int64_t work) {
  int64_t b = (work + kThreads - 1) / kThreads;
  int64_t cap = (int64_t)ctx->sm_count * 16;
  return (int)std::max<int64_t>(1, std::min(b, cap));
}

}  // namespace

// Shared driver.  d_data, d_idx are device pointers.  If `paired_out` is given, the
// bootstrap means/squares are written as the paired complex layout used by the
// estimator (z_p = M_2p + i M_2p+1, w_p = V_2p + i V_2p+1, zF = M_identity + 0i);
// otherwise plain G x nboot FP64 arrays (and/or the identity when nboot == 0).
struct DiracScales {
  double sm, sv;
};

static DiracScales dirac_core(pkde_ctx *ctx, const pkde_grid *g, const double *d_data, int64_t n,
                              const int32_t *d_idx, int64_t nboot, bool with_identity, uint64_t seed,
                              bool want_sq, double2 *paired_out, double *plain_m, double *plain_v,
                              uint32_t *d_counts_out, cudaStream_t st) {
  grid_validate(g);
  if (n < 1 || n >= (int64_t(1) << 31)) throw invalid("number of samples must be in [1, 2^31)");
  GridDev gd = to_dev(g);
  const int64_t G = grid_size(g);
  const int N = g->ndim;
  const int nc = 1 << N;
  const int64_t nslots = nboot + (with_identity ? 1 : 0);

  // scratch: cell (u32 n), rh (N*n f64), counts (nslots*G u32), q arrays (nc*n u64 x2), misc
  uint32_t *cell = (uint32_t *)ensure(ctx, BUF_PRE_CELL, sizeof(uint32_t) * n);
  double *rh = (double *)ensure(ctx, BUF_PRE_RH, sizeof(double) * N * n + sizeof(unsigned long long) * 2 * nc * n);
  unsigned long long *qm = reinterpret_cast<unsigned long long *>(rh + N * n);
  unsigned long long *qv = qm + (int64_t)nc * n;
  uint32_t *counts = (uint32_t *)ensure(ctx, BUF_COUNTS, sizeof(uint32_t) * nslots * G);
  int *misc = (int *)ensure(ctx, BUF_MISC, 256);
  int *err = misc;
  unsigned int *maxc = reinterpret_cast<unsigned int *>(misc + 1);
  int64_t *corner_off = reinterpret_cast<int64_t *>(misc + 8);  // 16 entries

  int64_t off_h[16];
  for (int c = 0; c < nc; ++c) {
    int64_t o = 0;
    for (int j = 0; j < N; ++j)
      if (!((c >> (N - 1 - j)) & 1)) o += gd.stride[j];
    off_h[c] = o;
  }
  PKDE_CUDA_TRY(cudaMemsetAsync(misc, 0, 64, st));
  PKDE_CUDA_TRY(cudaMemcpyAsync(corner_off, off_h, sizeof(int64_t) * nc, cudaMemcpyHostToDevice, st));
  PKDE_CUDA_TRY(cudaMemsetAsync(counts, 0, sizeof(uint32_t) * nslots * G, st));

  {
    ::pkde::Trace _tr(ctx, PKDE_PHASE_BINNING, st);
    prepass_kernel<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, st>>>(gd, d_data, n, cell, rh, err);
  }
  PKDE_CHECK_LAUNCH();
  {
    ::pkde::Trace _tr(ctx, PKDE_PHASE_BINNING, st);
    count_kernel<<<grid_blocks(ctx, nslots * n), kThreads, 0, st>>>(cell, n, nslots, nboot, G, d_idx, seed, counts, err);
  }
  PKDE_CHECK_LAUNCH();
  {
    ::pkde::Trace _tr(ctx, PKDE_PHASE_BINNING, st);
    max_kernel<<<grid_blocks(ctx, nslots * G), kThreads, 0, st>>>(counts, nslots * G, maxc);
  }
  PKDE_CHECK_LAUNCH();
  int hbuf[2];
  PKDE_CUDA_TRY(cudaMemcpyAsync(hbuf, misc, sizeof(int) * 2, cudaMemcpyDeviceToHost, st));
  PKDE_CUDA_TRY(cudaStreamSynchronize(st));
  if (hbuf[0] & 1) throw invalid("Data points lie beyond grid. Remove them or increase grid boundaries.");
  if (hbuf[0] & 2)
    throw invalid("Data points lie within one rounding of the upper grid bound. Remove them or increase grid boundaries.");
  if (hbuf[0] & 4) throw invalid("Bootstrap indices must lie in 1:n_samples.");
  const double cmax = (double)(uint32_t)hbuf[1];

  // term <= prod(h) / (n prod(h)^2); a cell sums at most 2^N * cmax terms.
  double sp = g->h[0];
  for (int j = 1; j < N; ++j) sp = sp * g->h[j];
  const double denom = (double)n * (sp * sp);
  const double tmax = (1.0 / ((double)n * sp)) * (1.0 + 1e-12);
  const double bound_m = (double)nc * std::max(cmax, 1.0) * tmax;
  const double bound_v = (double)nc * std::max(cmax, 1.0) * tmax * tmax;
  int ex_m, ex_v;
  std::frexp(bound_m, &ex_m);  // bound_m < 2^ex_m
  std::frexp(bound_v, &ex_v);
  const int e_m = 62 - ex_m;
  const int e_v = 62 - ex_v;

  {
    ::pkde::Trace _tr(ctx, PKDE_PHASE_BINNING, st);
    quantize_kernel<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, st>>>(gd, rh, n, denom, e_m, e_v, qm,
                                                                                     want_sq ? qv : nullptr);
  }
  PKDE_CHECK_LAUNCH();
  const double sm = std::ldexp(1.0, -e_m), sv = std::ldexp(1.0, -e_v);
  if (paired_out) {
    const int64_t npairs = (nboot + 1) / 2;
    unsigned long long *acc = reinterpret_cast<unsigned long long *>(paired_out);
    PKDE_CUDA_TRY(cudaMemsetAsync(acc, 0, sizeof(double2) * (2 * npairs + 1) * G, st));
    {
      ::pkde::Trace _tr(ctx, PKDE_PHASE_BINNING, st);
      weight_kernel<true><<<grid_blocks(ctx, nslots * n), kThreads, 0, st>>>(
          cell, n, nslots, nboot, G, N, corner_off, d_idx, seed, qm, want_sq ? qv : nullptr, acc, nullptr, npairs, err);
    }
    PKDE_CHECK_LAUNCH();
    {
      ::pkde::Trace _tr(ctx, PKDE_PHASE_BINNING, st);
      dequant_paired_kernel<<<grid_blocks(ctx, (2 * npairs + 1) * G * 2), kThreads, 0, st>>>(acc, G, npairs, sm, sv);
    }
    PKDE_CHECK_LAUNCH();
  } else {
    unsigned long long *am = reinterpret_cast<unsigned long long *>(plain_m);
    unsigned long long *av = reinterpret_cast<unsigned long long *>(plain_v);
    PKDE_CUDA_TRY(cudaMemsetAsync(am, 0, sizeof(double) * nslots * G, st));
    if (av) PKDE_CUDA_TRY(cudaMemsetAsync(av, 0, sizeof(double) * nboot * G, st));
    {
      ::pkde::Trace _tr(ctx, PKDE_PHASE_BINNING, st);
      weight_kernel<false><<<grid_blocks(ctx, nslots * n), kThreads, 0, st>>>(
          cell, n, nslots, nboot, G, N, corner_off, d_idx, seed, qm, (want_sq && av) ? qv : nullptr, am, av, 0, err);
    }
    PKDE_CHECK_LAUNCH();
    {
      ::pkde::Trace _tr(ctx, PKDE_PHASE_BINNING, st);
      dequant_kernel<<<grid_blocks(ctx, nslots * G), kThreads, 0, st>>>(am, nslots * G, sm);
    }
    PKDE_CHECK_LAUNCH();
    if (av) {
      {
        ::pkde::Trace _tr(ctx, PKDE_PHASE_BINNING, st);
        dequant_kernel<<<grid_blocks(ctx, nboot * G), kThreads, 0, st>>>(av, nboot * G, sv);
      }
      PKDE_CHECK_LAUNCH();
    }
  }
  if (d_counts_out) PKDE_CUDA_TRY(cudaMemcpyAsync(d_counts_out, counts, sizeof(uint32_t) * nslots * G,
                                                  cudaMemcpyDeviceToDevice, st));
  return DiracScales{sm, sv};
}

// Estimator entry: paired spectra-ready layout (nboot resamples + identity), in two
// phases around one host read-back of the error flags and the largest count, so that
// the estimations of a batch share one synchronisation.
size_t dirac_job_scratch(const pkde_grid *g, int64_t n, int64_t nboot) {
  const int N = g->ndim;
  const int64_t nc = int64_t(1) << N;
  const int64_t G = grid_size(g);
  const int64_t nchunk = (G + kScanChunk - 1) / kScanChunk;
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const int64_t npairs = (nboot + 1) / 2;
  return al(sizeof(uint32_t) * n) + al(sizeof(double) * N * n + sizeof(unsigned long long) * 4 * nc * n) +
         al(sizeof(uint32_t) * (nboot + 1) * G) + 2 * al(sizeof(uint32_t) * n) + 2 * al(sizeof(uint32_t) * G) +
         al(sizeof(uint32_t) * nchunk) + al(sizeof(uint32_t) * std::max<int64_t>(nboot, 1) * n) +
         al(sizeof(double2) * (2 * npairs + 1) * G);
}

void dirac_job_bind(DiracJob &j, char *scratch, int *misc) {
  const int N = j.g->ndim;
  const int64_t nc = int64_t(1) << N;
  const int64_t G = grid_size(j.g);
  const int64_t nchunk = (G + kScanChunk - 1) / kScanChunk;
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  j.cell = (uint32_t *)scratch;
  scratch += al(sizeof(uint32_t) * j.n);
  j.rh = (double *)scratch;
  j.qm_lo = reinterpret_cast<long long *>(j.rh + N * j.n) + 2 * nc * j.n;  // after the high parts
  j.qv_lo = j.qm_lo + nc * j.n;
  scratch += al(sizeof(double) * N * j.n + sizeof(unsigned long long) * 4 * nc * j.n);
  j.counts = (uint32_t *)scratch;  // draws per lower cell and resample (slot nboot: identity)
  scratch += al(sizeof(uint32_t) * (j.nboot + 1) * G);
  j.pos = (uint32_t *)scratch;
  scratch += al(sizeof(uint32_t) * j.n);
  j.cell_sorted = (uint32_t *)scratch;
  scratch += al(sizeof(uint32_t) * j.n);
  j.cstart = (uint32_t *)scratch;
  scratch += al(sizeof(uint32_t) * G);
  j.cfill = (uint32_t *)scratch;
  scratch += al(sizeof(uint32_t) * G);
  j.csum = (uint32_t *)scratch;
  scratch += al(sizeof(uint32_t) * nchunk);
  j.mult = (uint32_t *)scratch;
  scratch += al(sizeof(uint32_t) * std::max<int64_t>(j.nboot, 1) * j.n);
  j.acc_lo = (unsigned long long *)scratch;
  j.misc = misc;
}

// Phase A: bounds check and cell pre-pass, exact counts, largest count (misc[0] error
// bits, misc[1] max count).  Nothing is read back here.
void dirac_job_phase_a(pkde_ctx *ctx, DiracJob &j, cudaStream_t st) {
  const pkde_grid *g = j.g;
  grid_validate(g);
  const int64_t n = j.n;
  if (n < 1 || n >= (int64_t(1) << 31)) throw invalid("number of samples must be in [1, 2^31)");
  GridDev gd = to_dev(g);
  const int64_t G = grid_size(g);
  const int N = g->ndim;
  const int nc = 1 << N;
  const int64_t nslots = j.nboot + 1;
  int *misc = j.misc;
  unsigned int *maxc = reinterpret_cast<unsigned int *>(misc + 1);
  int64_t *corner_off = reinterpret_cast<int64_t *>(misc + 8);  // 16 entries
  for (int c = 0; c < nc; ++c) {
    int64_t o = 0;
    for (int q = 0; q < N; ++q)
      if (!((c >> (N - 1 - q)) & 1)) o += gd.stride[q];
    j.corner_off_h[c] = o;
  }
  PKDE_CUDA_TRY(cudaMemsetAsync(misc, 0, 64, st));
  PKDE_CUDA_TRY(cudaMemcpyAsync(corner_off, j.corner_off_h, sizeof(int64_t) * nc, cudaMemcpyHostToDevice, st));
  PKDE_CUDA_TRY(cudaMemsetAsync(j.counts, 0, sizeof(uint32_t) * nslots * G, st));
  {
    ::pkde::Trace _tr(ctx, PKDE_PHASE_BINNING, st);
    prepass_kernel<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, st>>>(gd, j.d_data, n, j.cell, j.rh,
                                                                                    misc);
  }
  PKDE_CHECK_LAUNCH();
  {
    // samples per lower cell (the identity slot); the resamples' counts are summed from
    // their multiplicities once the samples are in cell order
    ::pkde::Trace _tr(ctx, PKDE_PHASE_BINNING, st);
    count_kernel<<<grid_blocks(ctx, n), kThreads, 0, st>>>(j.cell, n, 1, 0, G, nullptr, 0, j.counts + j.nboot * G,
                                                          misc);
  }
  PKDE_CHECK_LAUNCH();
  // samples in lower-cell order (counting sort from the identity counts), then each
  // resample's draws as per-sample multiplicities in that order
  const uint32_t *idc = j.counts + j.nboot * G;
  const int64_t nchunk = (G + kScanChunk - 1) / kScanChunk;
  {
    ::pkde::Trace _tr(ctx, PKDE_PHASE_BINNING, st);
    cell_chunk_sum_kernel<<<(unsigned)nchunk, kThreads, 0, st>>>(idc, G, j.csum);
  }
  PKDE_CHECK_LAUNCH();
  {
    ::pkde::Trace _tr(ctx, PKDE_PHASE_BINNING, st);
    chunk_scan_kernel<<<1, 32, 0, st>>>(j.csum, nchunk);
  }
  PKDE_CHECK_LAUNCH();
  {
    ::pkde::Trace _tr(ctx, PKDE_PHASE_BINNING, st);
    cell_start_kernel<<<(unsigned)nchunk, kThreads, 0, st>>>(idc, G, j.csum, j.cstart, j.cfill);
  }
  PKDE_CHECK_LAUNCH();
  {
    ::pkde::Trace _tr(ctx, PKDE_PHASE_BINNING, st);
    cell_sort_kernel<<<grid_blocks(ctx, n), kThreads, 0, st>>>(j.cell, n, j.cstart, j.cfill, j.pos, j.cell_sorted);
  }
  PKDE_CHECK_LAUNCH();
  if (j.nboot > 0) {
    PKDE_CUDA_TRY(cudaMemsetAsync(j.mult, 0, sizeof(uint32_t) * j.nboot * n, st));
    {
      ::pkde::Trace _tr(ctx, PKDE_PHASE_BINNING, st);
      mult_kernel<<<grid_blocks(ctx, j.nboot * n), kThreads, 0, st>>>(n, j.nboot, j.d_idx, j.seed, j.pos, j.mult,
                                                                     misc);
    }
    PKDE_CHECK_LAUNCH();
  }
  if (j.nboot > 0) {
    ::pkde::Trace _tr(ctx, PKDE_PHASE_BINNING, st);
    resample_count_kernel<<<grid_blocks(ctx, j.nboot * n), kThreads, 0, st>>>(j.cell_sorted, n, j.nboot, G, j.mult,
                                                                              j.counts);
  }
  PKDE_CHECK_LAUNCH();
  {
    ::pkde::Trace _tr(ctx, PKDE_PHASE_BINNING, st);
    max_kernel<<<grid_blocks(ctx, nslots * G), kThreads, 0, st>>>(j.counts, nslots * G, maxc);
  }
  PKDE_CHECK_LAUNCH();
}

// Phase B, given misc[0..1] read back: error check, fixed-point scales, quantised
// corner terms, scatter into the paired spectra slots, conversion to FP64.
void binning_flags_check(const int *hmisc) {
  if (hmisc[0] & 1) throw invalid("Data points lie beyond grid. Remove them or increase grid boundaries.");
  if (hmisc[0] & 2)
    throw invalid("Data points lie within one rounding of the upper grid bound. Remove them or increase grid boundaries.");
  if (hmisc[0] & 4) throw invalid("Bootstrap indices must lie in 1:n_samples.");
}

void dirac_job_phase_b(pkde_ctx *ctx, DiracJob &j, const int *hmisc, cudaStream_t st) {
  const pkde_grid *g = j.g;
  if (hmisc) binning_flags_check(hmisc);
  GridDev gd = to_dev(g);
  const int64_t G = grid_size(g);
  const int N = g->ndim;
  const int nc = 1 << N;
  const int64_t n = j.n;
  const int64_t nboot = j.nboot;
  const int64_t nslots = nboot + 1;
  unsigned long long *qm = reinterpret_cast<unsigned long long *>(j.rh + N * n);
  unsigned long long *qv = qm + (int64_t)nc * n;
  const int64_t *corner_off = reinterpret_cast<const int64_t *>(j.misc + 8);
  int *esc = j.misc + 48;
  // term <= prod(h) / (n prod(h)^2); a cell sums at most 2^N * cmax terms.
  double sp = g->h[0];
  for (int q = 1; q < N; ++q) sp = sp * g->h[q];
  const double denom = (double)n * (sp * sp);
  const double tmax = (1.0 / ((double)n * sp)) * (1.0 + 1e-12);
  {
    ::pkde::Trace _tr(ctx, PKDE_PHASE_BINNING, st);
    scale_exponents_kernel<<<1, 32, 0, st>>>(j.misc, (double)nc, tmax, esc);
  }
  PKDE_CHECK_LAUNCH();
  {
    ::pkde::Trace _tr(ctx, PKDE_PHASE_BINNING, st);
    quantize_sorted_kernel<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, st>>>(gd, j.rh, n, denom, esc,
                                                                                            j.pos, qm, qv, j.qm_lo,
                                                                                            j.qv_lo);
  }
  PKDE_CHECK_LAUNCH();
  const int64_t npairs = (nboot + 1) / 2;
  unsigned long long *acc = reinterpret_cast<unsigned long long *>(j.paired_out);
  PKDE_CUDA_TRY(cudaMemsetAsync(acc, 0, sizeof(double2) * (2 * npairs + 1) * G, st));
  PKDE_CUDA_TRY(cudaMemsetAsync(j.acc_lo, 0, sizeof(double2) * (2 * npairs + 1) * G, st));
  {
    ::pkde::Trace _tr(ctx, PKDE_PHASE_BINNING, st);
    // resamples in chunks of at most 16, as even as possible (65 = 5 x 13, 33 = 3 x 11)
    const int64_t nchunk = (nslots + 15) / 16;
    const int BC = (int)((nslots + nchunk - 1) / nchunk);
    const int blocks = grid_blocks(ctx, nchunk * n);
#define PKDE_WS(NN)                                                                                          \
  weight_sorted_kernel<NN><<<blocks, kThreads, 0, st>>>(j.cell_sorted, n, nboot, G, corner_off, j.mult, qm, qv,   \
                                                        j.qm_lo, j.qv_lo, acc, j.acc_lo, npairs, BC, nchunk)
    switch (N) {
      case 1: PKDE_WS(1); break;
      case 2: PKDE_WS(2); break;
      case 3: PKDE_WS(3); break;
      default: PKDE_WS(4); break;
    }
#undef PKDE_WS
  }
  PKDE_CHECK_LAUNCH();
  {
    ::pkde::Trace _tr(ctx, PKDE_PHASE_BINNING, st);
    dequant_paired_esc_kernel<<<grid_blocks(ctx, (2 * npairs + 1) * G * 2), kThreads, 0, st>>>(acc, j.acc_lo, G,
                                                                                                npairs, esc);
  }
  PKDE_CHECK_LAUNCH();
}

}  // namespace pkde

extern "C" int pkde_dirac_sequence(pkde_ctx *ctx, const pkde_grid *grid, const double *data, int64_t n,
                                   const int32_t *boot_idx, int32_t nboot, uint64_t seed, double *means_out,
                                   double *sq_out, uint32_t *counts_out, uint32_t flags, void *stream) {
  return pkde_guard(ctx, [&] {
    using namespace pkde;
    if (!ctx) throw invalid("context is NULL");
    PKDE_CUDA_TRY(cudaSetDevice(ctx->device));
    settle_pending(ctx);
    cudaStream_t st = (cudaStream_t)stream;
    DrainOnError drain{ctx, st};
    grid_validate(grid);
    if (nboot < 0) throw invalid("Number of bootstraps must be non-negative");
    if (!data) throw invalid("data is NULL");
    const bool din = flags & PKDE_DEVICE_INPUT, dout = flags & PKDE_DEVICE_OUTPUT;
    const int N = grid->ndim;
    const int64_t G = grid_size(grid);
    const bool identity = nboot == 0;
    const int64_t nb = identity ? 0 : nboot;
    const int64_t nslots = identity ? 1 : nb;
    double *d_data = (double *)ensure(ctx, BUF_DATA, sizeof(double) * N * n);
    copy_in(d_data, data, sizeof(double) * N * n, din, st);
    int32_t *d_idx = nullptr;
    if (!identity && boot_idx) {
      d_idx = (int32_t *)ensure(ctx, BUF_IDX, sizeof(int32_t) * n * nb);
      copy_in(d_idx, boot_idx, sizeof(int32_t) * n * nb, din, st);
    }
    double *om = (double *)ensure(ctx, BUF_OUT, sizeof(double) * (2 * nslots * G) + sizeof(uint32_t) * nslots * G);
    double *ov = om + nslots * G;
    uint32_t *oc = reinterpret_cast<uint32_t *>(ov + nslots * G);
    dirac_core(ctx, grid, d_data, n, d_idx, nb, identity, seed, sq_out != nullptr && !identity, nullptr, om,
               (sq_out && !identity) ? ov : nullptr, oc, st);
    if (means_out) copy_out(means_out, om, sizeof(double) * nslots * G, dout, st);
    if (sq_out && !identity) copy_out(sq_out, ov, sizeof(double) * nslots * G, dout, st);
    if (sq_out && identity) {
      if (dout) PKDE_CUDA_TRY(cudaMemsetAsync(sq_out, 0, sizeof(double) * G, st));
      else std::memset(sq_out, 0, sizeof(double) * G);
    }
    if (counts_out) copy_out(counts_out, oc, sizeof(uint32_t) * nslots * G, dout, st);
    PKDE_CUDA_TRY(cudaStreamSynchronize(st));
  });
}

// ---------------------------------------------------------------------------------
// Binning without device allocation (pkde_dirac_sequence_noalloc).
//
// For callers that cannot allocate device memory -- a host framework whose caching
// allocator owns all of the GPU's memory, or a caller that must not call
// cudaMalloc/cudaFree (both synchronise the whole device and stall its other streams).
// The call itself is still blocking: it synchronises the caller's stream twice (the
// error flags and largest count are read back between the counting and the weighting
// phases, and the call waits for its end).  Scratch lives in one file-scope device array
// of fixed size; the caller passes only its input and output buffers.
// The limits below are the array's capacity.  Every call shares the array and it keeps
// the last call's contents, so what must start at zero is cleared on each call, and two
// calls whose work overlaps on the GPU (different streams, or host threads without
// ordering) race on it.
// ---------------------------------------------------------------------------------
namespace pkde {
namespace {

constexpr int64_t kNoAllocMaxSamples = 16384;     // samples per call
constexpr int64_t kNoAllocMaxCounts = 1 << 20;    // resamples x grid points, when counts_out is NULL
constexpr size_t kNoAllocCellBytes = sizeof(uint32_t) * kNoAllocMaxSamples;
constexpr size_t kNoAllocRhBytes = sizeof(double) * 4 * kNoAllocMaxSamples;
constexpr size_t kNoAllocQBytes = sizeof(unsigned long long) * 2 * 16 * kNoAllocMaxSamples;
constexpr size_t kNoAllocCountBytes = sizeof(uint32_t) * kNoAllocMaxCounts;
constexpr size_t kNoAllocMiscBytes = 256;
constexpr size_t kNoAllocBytes =
    kNoAllocCellBytes + kNoAllocRhBytes + kNoAllocQBytes + kNoAllocCountBytes + kNoAllocMiscBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of g_noalloc_scratch, looked up once per device (the name is only a
// host-side stand-in in host code).
constexpr int kNoAllocMaxDevices = 64;
unsigned char *g_noalloc_addr[kNoAllocMaxDevices] = {};
std::mutex g_noalloc_mu;

int noalloc_blocks(int sms, int64_t work) {
  const int64_t b = (work + kThreads - 1) / kThreads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)sms * 16));
}

unsigned char *noalloc_scratch_for_current_device() {
  int dev = 0;
  PKDE_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) throw invalid("device index %d beyond the supported range", dev);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void *p = nullptr;
    PKDE_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_addr[dev] = static_cast<unsigned char *>(p);
  }
  return g_noalloc_addr[dev];
}

}  // namespace
}  // namespace pkde

extern "C" int pkde_dirac_sequence_noalloc(pkde_ctx *ctx, const pkde_grid *grid, const double *data, int64_t n,
                                           const int32_t *boot_idx, int32_t nboot, uint64_t seed,
                                           double *means_out, double *sq_out, uint32_t *counts_out, void *stream) {
  return pkde_guard(ctx, [&] {
    using namespace pkde;
    grid_validate(grid);
    if (!data || !means_out) throw invalid("data and means_out are required (device pointers)");
    if (nboot < 0) throw invalid("Number of bootstraps must be non-negative");
    if (n < 1 || n > kNoAllocMaxSamples)
      throw invalid("pkde_dirac_sequence_noalloc: %lld samples, the limit is %lld", (long long)n,
                    (long long)kNoAllocMaxSamples);
    const int N = grid->ndim;
    const int nc = 1 << N;
    const int64_t G = grid_size(grid);
    const bool identity = nboot == 0;
    const int64_t nb = identity ? 0 : nboot;
    const int64_t nslots = identity ? 1 : nb;
    if (!counts_out && nslots * G > kNoAllocMaxCounts)
      throw invalid("pkde_dirac_sequence_noalloc: %lld resample x grid counters exceed the limit %lld (pass counts_out)",
                    (long long)(nslots * G), (long long)kNoAllocMaxCounts);
    cudaStream_t st = (cudaStream_t)stream;
    // the work runs on the device that owns the stream (the legacy default stream: the
    // calling thread's current device), which is made current for the call
    int dev = 0, sms = 1, prev = 0;
    PKDE_CUDA_TRY(cudaGetDevice(&prev));
    dev = prev;
    if (st) PKDE_CUDA_TRY(cudaStreamGetDevice(st, &dev));
    struct RestoreDevice {
      int d;
      bool on;
      ~RestoreDevice() {
        if (on) cudaSetDevice(d);
      }
    } restore{prev, dev != prev};
    if (dev != prev) PKDE_CUDA_TRY(cudaSetDevice(dev));
    DrainOnError drain{ctx, st};
    unsigned char *base = noalloc_scratch_for_current_device();
    PKDE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    uint32_t *cell = reinterpret_cast<uint32_t *>(base);
    double *rh = reinterpret_cast<double *>(base + kNoAllocCellBytes);
    unsigned long long *qm = reinterpret_cast<unsigned long long *>(base + kNoAllocCellBytes + kNoAllocRhBytes);
    unsigned long long *qv = qm + (int64_t)16 * kNoAllocMaxSamples;
    uint32_t *counts = counts_out ? counts_out
                                  : reinterpret_cast<uint32_t *>(base + kNoAllocCellBytes + kNoAllocRhBytes +
                                                                 kNoAllocQBytes);
    int *misc = reinterpret_cast<int *>(base + kNoAllocCellBytes + kNoAllocRhBytes + kNoAllocQBytes +
                                        kNoAllocCountBytes);
    int *err = misc;
    unsigned int *maxc = reinterpret_cast<unsigned int *>(misc + 1);
    int64_t *corner_off = reinterpret_cast<int64_t *>(misc + 8);
    GridDev gd = to_dev(grid);
    int64_t off_h[16];
    for (int c = 0; c < nc; ++c) {
      int64_t o = 0;
      for (int j = 0; j < N; ++j)
        if (!((c >> (N - 1 - j)) & 1)) o += gd.stride[j];
      off_h[c] = o;
    }
    // scratch keeps the previous call's contents: clear what must start at zero
    PKDE_CUDA_TRY(cudaMemsetAsync(misc, 0, 64, st));
    PKDE_CUDA_TRY(cudaMemcpyAsync(corner_off, off_h, sizeof(int64_t) * nc, cudaMemcpyHostToDevice, st));
    PKDE_CUDA_TRY(cudaMemsetAsync(counts, 0, sizeof(uint32_t) * nslots * G, st));
    const unsigned nblk = (unsigned)((n + kThreads - 1) / kThreads);
    prepass_kernel<<<nblk, kThreads, 0, st>>>(gd, data, n, cell, rh, err);
    PKDE_CHECK_LAUNCH();
    count_kernel<<<noalloc_blocks(sms, nslots * n), kThreads, 0, st>>>(cell, n, nslots, nb, G, boot_idx,
                                                                                      seed, counts, err);
    PKDE_CHECK_LAUNCH();
    max_kernel<<<noalloc_blocks(sms, nslots * G), kThreads, 0, st>>>(counts, nslots * G, maxc);
    PKDE_CHECK_LAUNCH();
    int hbuf[2];
    PKDE_CUDA_TRY(cudaMemcpyAsync(hbuf, misc, sizeof(int) * 2, cudaMemcpyDeviceToHost, st));
    PKDE_CUDA_TRY(cudaStreamSynchronize(st));
    if (hbuf[0] & 1) throw invalid("Data points lie beyond grid. Remove them or increase grid boundaries.");
    if (hbuf[0] & 2)
      throw invalid("Data points lie within one rounding of the upper grid bound. Remove them or increase grid boundaries.");
    if (hbuf[0] & 4) throw invalid("Bootstrap indices must lie in 1:n_samples.");
    const double cmax = (double)(uint32_t)hbuf[1];
    double sp = grid->h[0];
    for (int j = 1; j < N; ++j) sp = sp * grid->h[j];
    const double denom = (double)n * (sp * sp);
    const double tmax = (1.0 / ((double)n * sp)) * (1.0 + 1e-12);
    int ex_m, ex_v;
    std::frexp((double)nc * std::max(cmax, 1.0) * tmax, &ex_m);
    std::frexp((double)nc * std::max(cmax, 1.0) * tmax * tmax, &ex_v);
    const int e_m = 62 - ex_m, e_v = 62 - ex_v;
    const bool want_sq = sq_out != nullptr && !identity;
    quantize_kernel<<<nblk, kThreads, 0, st>>>(gd, rh, n, denom, e_m, e_v, qm, want_sq ? qv : nullptr);
    PKDE_CHECK_LAUNCH();
    // the sums accumulate as 64-bit integers in the caller's output buffers
    unsigned long long *am = reinterpret_cast<unsigned long long *>(means_out);
    unsigned long long *av = want_sq ? reinterpret_cast<unsigned long long *>(sq_out) : nullptr;
    PKDE_CUDA_TRY(cudaMemsetAsync(am, 0, sizeof(double) * nslots * G, st));
    if (av) PKDE_CUDA_TRY(cudaMemsetAsync(av, 0, sizeof(double) * nb * G, st));
    weight_kernel<false><<<noalloc_blocks(sms, nslots * n), kThreads, 0, st>>>(
        cell, n, nslots, nb, G, N, corner_off, boot_idx, seed, qm, av ? qv : nullptr, am, av, 0, err);
    PKDE_CHECK_LAUNCH();
    dequant_kernel<<<noalloc_blocks(sms, nslots * G), kThreads, 0, st>>>(am, nslots * G,
                                                                                       std::ldexp(1.0, -e_m));
    PKDE_CHECK_LAUNCH();
    if (av) {
      dequant_kernel<<<noalloc_blocks(sms, nb * G), kThreads, 0, st>>>(av, nb * G, std::ldexp(1.0, -e_v));
      PKDE_CHECK_LAUNCH();
    }
    if (sq_out && identity) PKDE_CUDA_TRY(cudaMemsetAsync(sq_out, 0, sizeof(double) * G, st));
    PKDE_CUDA_TRY(cudaStreamSynchronize(st));
  });
}
