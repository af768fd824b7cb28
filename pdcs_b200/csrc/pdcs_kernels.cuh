// pdcs_kernels.cuh -- kernels of the PDHG hot path (FP64).
//
// One PDHG attempt (rpdhg_alg_gpu_gen_scaling.jl:680-765) runs as
//   spmv(G^T, y_lag)          -> aty                 [1 matrix pass]
//   update_project<Primal>    x = P_X(x_lag + tau*dec*(aty - c)), sum |dx|^2
//   spmv2(G, x, x_lag)        -> gx, gxl             [1 matrix pass, 2 gathers]
//   update_project<Dual>      y = P_Y(y_lag - sigma*dec*(2gx - gxl - h)),
//                             sum |dy|^2, sum dy*(gx - gxl)   (= dx' G' dy)
//   control                   eta_bar test, accept / retry, next step sizes
//   reflect                   aggressive extrapolation + eta-weighted averages
// The reference's third SpMV (G' dy, :712) is replaced by the identity
// dx' G' dy = dy' (G x - G x_lag), which the second pass provides for free.
#pragma once
#include <type_traits>

#include "pdcs_device.cuh"

namespace pdcs {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

enum AccKind : int32_t { ACC_SUM = 0, ACC_MAX = 1 };

// ---------------------------------------------------------------------------
// Device-resident solver state (one per solve).
// ---------------------------------------------------------------------------
enum HaltReason : int32_t {
  HALT_NONE = 0,
  HALT_CHECK = 1,          // attempt with iter % check_freq == 0: host runs the exit check
  HALT_RESTART_CHECK = 2,  // accepted step with iter % restart_freq == 0
  HALT_ARTIFICIAL = 3,     // inner >= beta_artificial * iter (or forced restart)
  HALT_LIMIT = 4,          // attempt limit reached
  HALT_RESOLVING_CHECK = 5,  // resolving mode: restart / exit tests due after this step
};

struct PdhgState {
  double eta, eta_p, eta_bar, omega, dec, dec_next, extra, eta_cum;
  double tau, sigma;   // params.tau / params.sigma of the last attempt
  double ps, ds;       // primal / dual step of the current attempt (tau*dec, sigma*dec)
  double refl_tmp, refl_inv, refl_eta, refl_cum, refl_extra;
  double sum_dx2, sum_dy2, sum_dgdy;
  long long iter, iter_stepsize, inner, reject_count;
  long long check_freq, restart_freq, attempt_limit;
  int32_t active, do_reflect, halt_reason, accepted;
  int32_t force_restart, restart_enabled;
  uint32_t done_ctas;  // CTAs of the dual step that have finished (last one runs the control step)
  int32_t resolving;   // fixed-step PDHG with uniform averaging (resolving_pessimistic_step!)
};

// Shared by the control kernel and the host (after a checkpoint):
// the bookkeeping after an accepted step (:752-753 return, then the main
// loop :854-866 and the next call's entry :667, :676).
__host__ __device__ inline void post_accept(PdhgState& st, bool force) {
  double eta_acc = st.eta > 1e-30 ? st.eta : 1e-30;
  st.inner += 1;
  double di = (double)st.inner;
  st.refl_tmp = (di + 1.0) / (di + 2.0);
  st.refl_inv = 1.0 / (di + 2.0);
  st.refl_eta = eta_acc;
  st.refl_cum = st.eta_cum;
  st.refl_extra = st.extra;
  st.eta_cum += eta_acc;
  st.do_reflect = 1;
  // next step call
  st.dec = st.dec_next;
  st.eta = st.eta_p > 1e-6 ? st.eta_p : 1e-6;
  st.reject_count = 0;
  st.ps = (st.eta / st.omega) * st.dec;
  st.ds = (st.eta * st.omega) * st.dec;
  bool artificial = ((double)st.inner >= (double)st.iter * 0.223 && st.iter > 10000) || (force && st.inner > 100);
  bool restart_due = st.restart_enabled && st.restart_freq > 0 && (st.iter % st.restart_freq == 0);
  if (artificial) {
    st.halt_reason = HALT_ARTIFICIAL;
    st.active = 0;
  } else if (restart_due) {
    st.halt_reason = HALT_RESTART_CHECK;
    st.active = 0;
  }
}

__host__ __device__ inline void after_reject(PdhgState& st) {
  st.eta = st.eta_p;
  st.reject_count += 1;
  st.ps = (st.eta / st.omega) * st.dec;
  st.ds = (st.eta * st.omega) * st.dec;
}

// ---------------------------------------------------------------------------
// CSR SpMV with rows binned by length.  Bin b < 6 holds rows handled by a
// group of g = 2^b lanes (rows of up to L g nonzeros for a schedule of L
// nonzeros per lane, picked per matrix by the setup autotuner); bin 6 holds
// longer rows, one CTA each; bin 7 (split rows: more than kSplitMin
// nonzeros) holds chunks of kSplitChunk nonzeros, a CTA per chunk, whose
// partial sums the row's last chunk to finish adds in chunk order.  One
// launch covers all bins: CTA ranges [cta0[b], cta0[b+1]).
// ---------------------------------------------------------------------------
constexpr int kBins = 8;
constexpr int kSplitBin = kBins - 1;
constexpr int kRowBin = kBins - 2;
constexpr int kSplitPer = 16;                        // nonzeros per thread of a chunk
constexpr int kSplitChunk = kSplitPer * kThreads;   // 4096
constexpr int64_t kSplitMin = 4 * kSplitChunk;      // rows of more nonzeros are split

// rows[q] for the q-th row in bin order: {row, first nonzero, end, instance};
// split-row chunks: {row, first nonzero, end, chunk slot} (slots numbered
// over all chunks, a row's chunks consecutive)
template <class T>
struct CsrT {
  int64_t m, n, nnz;
  const int32_t* rp;
  const int32_t* ci;
  const T* v;
  const int4* rows;          // row descriptors ordered by bin (one 16-byte load per row)
  const int64_t* dbin;       // device bin offsets (a compacted row list) or NULL: bin_off
  int32_t lane_nnz;          // schedule: at most lane_nnz nonzeros per lane in bins 0..5
  int64_t bin_off[kBins + 1];
  int32_t cta0[kBins + 1];   // first CTA of each bin, cta0[kBins] = grid size
  double* spart = nullptr;   // split rows: 2 partial sums per chunk slot
  unsigned* scnt = nullptr;  // split rows: finished chunks, at the row's first slot (reset to 0 by the last)
};
using CsrDev = CsrT<double>;

// Row sums in T.  FP32 rows use FP32 products and sums; the long-row bin
// (rows of more than 128 nonzeros, one CTA each) adds with Kahan compensation.
template <class T>
struct RowAcc {
  T s = T(0), c = T(0);
  __device__ __forceinline__ void add(T v) {
    if constexpr (std::is_same_v<T, float>) {
      const float y = v - c;
      const float t = s + y;
      c = (t - s) - y;
      s = t;
    } else {
      s += v;
    }
  }
};

// Vectors of one SpMV pass (NV): 1 (x0), 2 (x0 and x1, two arrays) or kPair
// (x0 holds the two vectors interleaved, x0[2 c] and x0[2 c + 1]: one gather
// of 2 T per nonzero instead of two gathers of T).
constexpr int kPair = 3;
template <class T> struct Vec2T;
template <> struct Vec2T<float> { using type = float2; };
template <> struct Vec2T<double> { using type = double2; };

template <int NV, class T>
__device__ __forceinline__ void spmv_gather(const T* __restrict__ x0, const T* __restrict__ x1, int32_t c, T& a,
                                            T& b) {
  if constexpr (NV == kPair) {
    const auto v = reinterpret_cast<const typename Vec2T<T>::type*>(x0)[c];
    a = v.x;
    b = v.y;
  } else {
    a = x0[c];
    b = NV == 2 ? x1[c] : T(0);
  }
}

// MASK: rows whose instance (rows[q].w) has imask == 0 are skipped (batched solver).
// LN = A.lane_nnz: a lane holds at most LN nonzeros of its row in bins 0..5, so
// all of a lane's value / index loads are issued together, then all its gathers.
template <int NV, bool MASK = false, class T = double, int LN = 4>
__global__ void __launch_bounds__(kThreads) spmv_binned_kernel(CsrT<T> A,
                                                              const std::type_identity_t<T>* __restrict__ x0,
                                                              const std::type_identity_t<T>* __restrict__ x1,
                                                              std::type_identity_t<T>* __restrict__ y0,
                                                              std::type_identity_t<T>* __restrict__ y1,
                                                              const int32_t* __restrict__ active,
                                                              int32_t* __restrict__ clear_flag = nullptr,
                                                              const uint8_t* __restrict__ imask = nullptr) {
  // first kernel of a PDHG attempt: the previous attempt's reflection (if any)
  // has run by now, so its flag is cleared here, before the halt check
  if (clear_flag && blockIdx.x == 0 && threadIdx.x == 0) *clear_flag = 0;
  if (active && !*active) return;
  const int cta = blockIdx.x;
  int bin = 0;
#pragma unroll
  for (int b = 1; b < kBins; ++b)
    if (cta >= A.cta0[b]) bin = b;
  const int64_t r0 = A.dbin ? A.dbin[bin] : A.bin_off[bin], r1 = A.dbin ? A.dbin[bin + 1] : A.bin_off[bin + 1];
  const int ncta = A.cta0[bin + 1] - A.cta0[bin];
  const int lcta = cta - A.cta0[bin];
  if (bin < kRowBin) {
    const int g = 1 << bin;
    const int lane_g = threadIdx.x & (g - 1);
    const int64_t rows_per_cta = kThreads / g;
    // the loop bound is uniform across the warp (all lanes reach the shuffles)
    const int64_t warp_first = r0 + (int64_t)lcta * rows_per_cta + (threadIdx.x >> 5) * (32 / g);
    for (int64_t qb = warp_first; qb < r1; qb += (int64_t)ncta * rows_per_cta) {
      const int64_t q = qb + (threadIdx.x & 31) / g;
      bool valid = q < r1;
      const int4 ri = valid ? __ldg(A.rows + q) : make_int4(0, 0, 0, 0);
      const int32_t row = ri.x;
      if (MASK && valid) valid = imask[ri.w] != 0;
      const int32_t kb = valid ? ri.y : 0, ke = valid ? ri.z : 0;
      T av[LN];
      int32_t cv[LN];
#pragma unroll
      for (int u = 0; u < LN; ++u) {
        const int32_t k = kb + lane_g + u * g;
        const bool ok = k < ke;
        av[u] = ok ? A.v[k] : T(0);
        cv[u] = ok ? A.ci[k] : -1;
      }
      T p0[4] = {T(0), T(0), T(0), T(0)}, p1[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll
      for (int u = 0; u < LN; ++u) {
        if (cv[u] >= 0) {
          T a, b;
          spmv_gather<NV>(x0, x1, cv[u], a, b);
          p0[u & 3] = fma(av[u], a, p0[u & 3]);
          if (NV >= 2) p1[u & 3] = fma(av[u], b, p1[u & 3]);
        }
      }
      T s0 = (p0[0] + p0[1]) + (p0[2] + p0[3]);
      T s1 = (p1[0] + p1[1]) + (p1[2] + p1[3]);
      for (int o = g >> 1; o > 0; o >>= 1) {
        s0 += __shfl_down_sync(kFull, s0, o, g);
        if (NV >= 2) s1 += __shfl_down_sync(kFull, s1, o, g);
      }
      if (valid && lane_g == 0) {
        y0[row] = s0;
        if (NV >= 2) y1[row] = s1;
      }
    }
  } else if (bin == kRowBin) {
    __shared__ T red0[kWarps], red1[kWarps];
    for (int64_t q = r0 + lcta; q < r1; q += ncta) {
      const int4 ri = __ldg(A.rows + q);
      const int32_t row = ri.x;
      if (MASK && !imask[ri.w]) continue;  // CTA-uniform
      const int32_t kb = ri.y, ke = ri.z;
      RowAcc<T> a0, a1;
      // four nonzeros per thread in flight: their loads, then their gathers
      for (int32_t kq = kb + threadIdx.x; kq < ke; kq += 4 * kThreads) {
        T av[4];
        int32_t cv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int32_t k = kq + u * kThreads;
          av[u] = k < ke ? A.v[k] : T(0);
          cv[u] = k < ke ? A.ci[k] : -1;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          if (cv[u] < 0) continue;
          T u0, u1;
          spmv_gather<NV>(x0, x1, cv[u], u0, u1);
          a0.add(av[u] * u0);
          if (NV >= 2) a1.add(av[u] * u1);
        }
      }
      T s0 = a0.s, s1 = a1.s;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_down_sync(kFull, s0, o);
        if (NV >= 2) s1 += __shfl_down_sync(kFull, s1, o);
      }
      const int w = threadIdx.x >> 5;
      if ((threadIdx.x & 31) == 0) {
        red0[w] = s0;
        red1[w] = s1;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        RowAcc<T> t0, t1;
        for (int i = 0; i < kWarps; ++i) {
          t0.add(red0[i]);
          t1.add(red1[i]);
        }
        y0[row] = t0.s;
        if (NV >= 2) y1[row] = t1.s;
      }
      __syncthreads();
    }
  } else if constexpr (!MASK) {
    // split rows: a chunk of kSplitChunk nonzeros per CTA, kSplitPer per thread
    // (all loads, then all gathers); products in T, the chunk's sum in FP64;
    // the chunk that finishes its row last adds the row's partials in chunk
    // order, so the result does not depend on which chunk finishes last
    __shared__ double sr0[kWarps], sr1[kWarps];
    __shared__ int last;
    for (int64_t q = r0 + lcta; q < r1; q += ncta) {
      const int4 ri = __ldg(A.rows + q);
      const int32_t row = ri.x, kb = ri.y, ke = ri.z, slot = ri.w;
      T av[kSplitPer];
      int32_t cv[kSplitPer];
#pragma unroll
      for (int u = 0; u < kSplitPer; ++u) {
        const int32_t k = kb + threadIdx.x + u * kThreads;
        av[u] = k < ke ? A.v[k] : T(0);
        cv[u] = k < ke ? A.ci[k] : -1;
      }
      T p0[4] = {T(0), T(0), T(0), T(0)}, p1[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll
      for (int u = 0; u < kSplitPer; ++u) {
        if (cv[u] >= 0) {
          T a, b;
          spmv_gather<NV>(x0, x1, cv[u], a, b);
          p0[u & 3] = fma(av[u], a, p0[u & 3]);
          if (NV >= 2) p1[u & 3] = fma(av[u], b, p1[u & 3]);
        }
      }
      double s0 = ((double)p0[0] + (double)p0[1]) + ((double)p0[2] + (double)p0[3]);
      double s1 = ((double)p1[0] + (double)p1[1]) + ((double)p1[2] + (double)p1[3]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_down_sync(kFull, s0, o);
        if (NV >= 2) s1 += __shfl_down_sync(kFull, s1, o);
      }
      if ((threadIdx.x & 31) == 0) {
        sr0[threadIdx.x >> 5] = s0;
        sr1[threadIdx.x >> 5] = s1;
      }
      __syncthreads();
      const int32_t rb = A.rp[row], re = A.rp[row + 1];
      const int32_t first = slot - (kb - rb) / kSplitChunk;
      const int32_t nch = (re - rb + kSplitChunk - 1) / kSplitChunk;
      if (threadIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0;
        for (int w = 0; w < kWarps; ++w) {
          t0 += sr0[w];
          t1 += sr1[w];
        }
        A.spart[2 * (int64_t)slot] = t0;
        A.spart[2 * (int64_t)slot + 1] = t1;
        __threadfence();
        last = atomicAdd(A.scnt + first, 1u) == (unsigned)(nch - 1);
      }
      __syncthreads();
      if (last && threadIdx.x < 32) {  // CTA-uniform branch into warp 0
        __threadfence();
        double t0 = 0.0, t1 = 0.0;
        for (int32_t c = threadIdx.x; c < nch; c += 32) {
          t0 += __ldcg(A.spart + 2 * (int64_t)(first + c));
          if (NV >= 2) t1 += __ldcg(A.spart + 2 * (int64_t)(first + c) + 1);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          t0 += __shfl_down_sync(kFull, t0, o);
          if (NV >= 2) t1 += __shfl_down_sync(kFull, t1, o);
        }
        if (threadIdx.x == 0) {
          y0[row] = (T)t0;
          if (NV >= 2) y1[row] = (T)t1;
          A.scnt[first] = 0u;
        }
      }
      __syncthreads();
    }
  }
}

// Launch spmv_binned_kernel with the matrix's schedule (A.lane_nnz).
template <int NV, bool MASK = false, class T>
inline void launch_spmv(const CsrT<T>& A, const std::type_identity_t<T>* x0, const std::type_identity_t<T>* x1,
                        std::type_identity_t<T>* y0, std::type_identity_t<T>* y1, const int32_t* active,
                        cudaStream_t s, int32_t* clear_flag = nullptr, const uint8_t* imask = nullptr) {
  const int grid = A.cta0[kBins];
  switch (A.lane_nnz) {
    case 1: spmv_binned_kernel<NV, MASK, T, 1><<<grid, kThreads, 0, s>>>(A, x0, x1, y0, y1, active, clear_flag, imask); break;
    case 2: spmv_binned_kernel<NV, MASK, T, 2><<<grid, kThreads, 0, s>>>(A, x0, x1, y0, y1, active, clear_flag, imask); break;
    case 8: spmv_binned_kernel<NV, MASK, T, 8><<<grid, kThreads, 0, s>>>(A, x0, x1, y0, y1, active, clear_flag, imask); break;
    case 16: spmv_binned_kernel<NV, MASK, T, 16><<<grid, kThreads, 0, s>>>(A, x0, x1, y0, y1, active, clear_flag, imask); break;
    default: spmv_binned_kernel<NV, MASK, T, 4><<<grid, kThreads, 0, s>>>(A, x0, x1, y0, y1, active, clear_flag, imask); break;
  }
}

// ---------------------------------------------------------------------------
// Block structure of one vector for projections.
// ---------------------------------------------------------------------------
constexpr int kCls = 6;
// Lane groups of the cone schedule: class c < kCls - 1 holds blocks of at most
// 2 << c elements, projected by cls_lanes(c) lanes with kClsEPL elements per lane
// (32 / cls_lanes(c) blocks per warp); the last class takes a warp per block.
constexpr int kClsEPL = 2;
__host__ __device__ constexpr int cls_lanes(int c) { return (2 << c) / kClsEPL < 1 ? 1 : (2 << c) / kClsEPL; }

struct ConeTable {
  int64_t len;
  int32_t nseg;
  int32_t seg_kind[3];
  int64_t seg_start[3], seg_len[3];
  const double* lo;  // BOX bounds (global index)
  const double* hi;
  int64_t nwc;               // SOC / RSOC blocks
  const int64_t* wc_start;
  const int32_t* wc_len;
  const int8_t* wc_kind;     // PK_SOC or PK_RSOC
  int64_t exp_base, exp_count;   // contiguous triples
  int32_t exp_kind;              // PK_EXP or PK_DEXP
  int64_t dexp_base, dexp_count;
  int32_t dexp_kind;
  const double* S;           // scaling (NULL: unscaled)
  double* rho_ws;            // per exp/dual-exp cone warm start of the root (NULL: none)
  // warp-cone schedule by size class: class c < kCls - 1 packs blocks of at
  // most 2 << c elements, 32 / cls_lanes(c) per warp; the last class (> 32) takes a
  // warp per block.  sched lists warp-cone indices class by class.
  const int64_t* sched;
  int64_t cls_off[kCls + 1];  // ranges of sched per class
  int64_t task0[kCls + 1];    // first warp task of each class; task0[kCls] = tasks
  double* soc_ws;             // per warp cone warm start of the weighted-SOC root (NULL: none)
  // Active work lists (batched solver's iteration graph; NULL: the whole table).
  // act_meta: [0] elementwise chunks, [1 .. kCls + 1] warp tasks per class
  // (as task0), [kCls + 2 .. 2 kCls + 2] ranges of act_sched (as cls_off),
  // [2 kCls + 3] exp / dual-exp cones in act_exp.
  const int2* act_chunk;      // elementwise chunks {first element, length <= kThreads}
  const int64_t* act_meta;
  const int64_t* act_sched;   // warp-cone indices, class by class
  const int32_t* act_exp;     // exp / dual-exp cone ordinals (0 .. exp_count + dexp_count)
  const int4* act_desc;       // with act_sched: per scheduled cone {start, length | RSOC << 30, cone,
                              // instance}, so a lane group reads one record (NULL: the wc_* tables)
  int64_t elem_total;        // sum of seg_len
  int32_t ctaA, ctaB, ctaC;  // CTAs for elementwise / warp cones / exp cones
  // Huge SOC / RSOC blocks (kHugeBlock elements or more, at most kMaxHuge per
  // table; none in the batched solver's tables): projected together by the
  // first ctaD CTAs of the launch, which meet at bounded barriers (huge_bar)
  // between the reductions of the Newton solve; they are not in sched.
  int32_t ctaD;
  int32_t nhuge;
  int64_t huge_start[2];
  int64_t huge_len[2];
  int32_t huge_rsoc[2];
  int64_t huge_wc[2];   // the block's warp-cone index (its soc_ws warm start)
  unsigned* huge_bar;   // {arrivals, generation}
  int32_t* huge_err;    // set when a CTA gave up waiting at a barrier
  double* huge_red;     // 2 x ctaD x 4 partial sums (two alternating sets)
  double2* huge_scr;    // per element of the huge blocks: {D_i^2 x_i^2, D_i} of the current projection
  int64_t huge_soff[2]; // block h's first element in huge_scr
};
constexpr int kMaxHuge = 2;
constexpr int64_t kHugeBlock = 16384;  // blocks of at least this many elements take part D
// part D CTAs: at most two per SM of a 148-SM B200, so every one of them is
// resident (the update kernels run at least 2 CTAs per SM: <= 128 registers)
constexpr int kHugeMaxCtas = 2 * 148;
inline int table_grid(const ConeTable& T) { return T.ctaA + T.ctaB + T.ctaC + T.ctaD; }

__device__ __forceinline__ double elem_proj(int32_t kind, double z, int64_t j, const ConeTable& T) {
  switch (kind) {
    case PK_ZERO: return 0.0;
    case PK_NONNEG: return fmax(z, 0.0);
    case PK_BOX: return fmin(fmax(z, T.lo[j]), T.hi[j]);
    default: return z;
  }
}

template <int N>
__device__ inline void block_reduce_store(double (&acc)[N], const int32_t* kinds, double* partials, int nblocks) {
  __shared__ double sh[N][kWarps];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    double v = acc[k];
    if (kinds[k] == ACC_MAX) {
      for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(kFull, v, o));
    } else {
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
    }
    if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < N) {
    int k = threadIdx.x;
    double v = sh[k][0];
    for (int w = 1; w < kWarps; ++w) v = (kinds[k] == ACC_MAX) ? fmax(v, sh[k][w]) : v + sh[k][w];
    partials[(int64_t)k * nblocks + blockIdx.x] = v;
  }
}

// The control step of one PDHG attempt (rpdhg_alg_gpu_gen_scaling.jl:711-765)
// given the step's sums a = |dx|^2, b = |dy|^2, c = dy'(G x - G x_lag): form
// eta_bar and eta', decide accept / retry / halt.  Shared by the single-
// instance control block and the per-instance control of the batched solver.
__device__ inline void control_step(PdhgState& s, double a, double b, double c) {
  s.sum_dx2 = a;
  s.sum_dy2 = b;
  s.sum_dgdy = c;
  s.do_reflect = 0;
  double num = s.omega * s.sum_dx2 + s.sum_dy2 / s.omega;
  double den = 2.0 * fabs(s.sum_dgdy);
  s.eta_bar = num / (den + 1e-20);
  s.iter += 1;
  s.iter_stepsize += 1;
  double k1 = (double)(s.iter_stepsize + 1);
  s.eta_p = fmin((1.0 - pow(k1, -0.3)) * s.eta_bar, (1.0 + pow(k1, -0.6)) * s.eta);
  if (s.resolving) {
    // pdhg_one_iter_diagonal_rescaling! + average_seq (rpdhg_alg_gpu_gen_scaling.jl:250-263,
    // :561-568): every step is kept; x_lag <- x and the mean is the uniform average
    s.accepted = 1;
    s.inner += 1;
    s.refl_tmp = 1.0;
    s.refl_inv = 0.0;
    s.refl_extra = 0.0;
    s.refl_eta = 1.0;
    s.refl_cum = (double)s.inner;
    s.do_reflect = 1;
    bool due = (s.check_freq > 0 && s.iter % s.check_freq == 0) ||
               (s.restart_enabled && s.restart_freq > 0 && s.iter % s.restart_freq == 0);
    if (due) {
      s.halt_reason = HALT_RESOLVING_CHECK;
      s.active = 0;
    } else if (s.attempt_limit > 0 && s.iter >= s.attempt_limit) {
      s.halt_reason = HALT_LIMIT;
      s.active = 0;
    }
    return;
  }
  s.tau = s.eta / s.omega;
  s.sigma = s.eta * s.omega;
  s.accepted = (s.eta <= s.eta_bar) ? 1 : 0;
  if (s.check_freq > 0 && s.iter % s.check_freq == 0) {
    s.halt_reason = HALT_CHECK;  // the host runs the exit check, then decides
    s.active = 0;
  } else if (s.attempt_limit > 0 && s.iter >= s.attempt_limit) {
    s.halt_reason = HALT_LIMIT;
    s.active = 0;
  } else if (s.accepted) {
    post_accept(s, false);
  } else {
    after_reject(s);
    if (s.reject_count > 1000000) {
      s.eta = s.eta_p;  // the forced return hands back the last eta (:757-764)
      post_accept(s, true);
    }
  }
}

// Reduce the step's partial sums (fixed order) and run control_step; one CTA of kThreads threads.
__device__ inline void control_block(PdhgState* st, const double* px, int nbx, const double* py, int nby) {
  __shared__ double sh[3][kThreads];
  double a = 0.0, b = 0.0, c = 0.0;
  for (int i = threadIdx.x; i < nbx; i += kThreads) a += __ldcg(px + i);
  for (int i = threadIdx.x; i < nby; i += kThreads) {
    b += __ldcg(py + i);
    c += __ldcg(py + nby + i);
  }
  sh[0][threadIdx.x] = a;
  sh[1][threadIdx.x] = b;
  sh[2][threadIdx.x] = c;
  __syncthreads();
  for (int s2 = kThreads / 2; s2 > 0; s2 >>= 1) {
    if (threadIdx.x < s2) {
      sh[0][threadIdx.x] += sh[0][threadIdx.x + s2];
      sh[1][threadIdx.x] += sh[1][threadIdx.x + s2];
      sh[2][threadIdx.x] += sh[2][threadIdx.x + s2];
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  PdhgState s = *st;
  s.done_ctas = 0;
  control_step(s, sh[0][0], sh[1][0], sh[2][0]);
  *st = s;
}

// Barrier of the CTAs [0, n) of a launch (part D).  Every CTA of the launch's
// part D is resident: they have the lowest block indices, their number is at
// most the SM count, and no other CTA of the launch waits.  The wait is still
// bounded: a CTA that polls 2^24 times without the generation moving sets *err
// and gives up (the solve then reports a CUDA error instead of hanging).
__device__ inline bool huge_barrier(unsigned* bar, unsigned n, int32_t* err) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    __threadfence();
    const unsigned gen = *((volatile unsigned*)(bar + 1));
    if (atomicAdd(bar, 1u) == n - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      long long it = 0;
      while (*((volatile unsigned*)(bar + 1)) == gen) {
        if (++it > (1ll << 24) || *((volatile int32_t*)err)) {
          atomicExch(err, 1);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok != 0;
}

// Block-wide sums / maxima of NR values (every thread receives the results).
template <int NR>
__device__ inline void block_reduce_n(double (&v)[NR], const bool (&is_max)[NR]) {
  __shared__ double sh[NR][kWarps];
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    double x = v[r];
    for (int o = 16; o > 0; o >>= 1) {
      const double y = __shfl_xor_sync(kFull, x, o);
      x = is_max[r] ? fmax(x, y) : x + y;
    }
    if ((threadIdx.x & 31) == 0) sh[r][threadIdx.x >> 5] = x;
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    double x = sh[r][0];
    for (int w = 1; w < kWarps; ++w) x = is_max[r] ? fmax(x, sh[r][w]) : x + sh[r][w];
    v[r] = x;
  }
  __syncthreads();
}

// One reduction round of part D: this CTA's NR values go to its slot of the
// round's buffer; after the barrier warp 0 of every CTA combines the slots
// (lane l takes slots l, l + 32, ..., then a butterfly), the same operations in
// the same order in every CTA, so all CTAs hold bit-identical results.
// Returns false if a wait gave up.
template <int NR>
__device__ inline bool huge_allreduce(const ConeTable& T, int cta, int& round, double (&v)[NR],
                                      const bool (&is_max)[NR]) {
  __shared__ double res[NR];
  block_reduce_n<NR>(v, is_max);
  double* buf = T.huge_red + (size_t)(round & 1) * T.ctaD * 4;
  if (threadIdx.x < NR) buf[cta * 4 + threadIdx.x] = v[threadIdx.x];
  round++;
  if (!huge_barrier(T.huge_bar, (unsigned)T.ctaD, T.huge_err)) return false;
  if (threadIdx.x < 32) {
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      const double id = is_max[r] ? -__longlong_as_double(0x7ff0000000000000ll) : 0.0;
      double x = id;
#pragma unroll 4
      for (int c = threadIdx.x; c < T.ctaD; c += 32) {
        const double y = __ldcg(buf + c * 4 + r);
        x = is_max[r] ? fmax(x, y) : x + y;
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double y = __shfl_xor_sync(kFull, x, o);
        x = is_max[r] ? fmax(x, y) : x + y;
      }
      if (threadIdx.x == 0) res[r] = x;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < NR; ++r) v[r] = res[r];
  return true;
}

// Projection of huge block h of T (SOC, or RSOC through the rotation onto a
// weighted SOC) by the ctaD CTAs of part D together: CTA `cta` owns a
// contiguous slice of the block (elements 0 and 1 in CTA 0), the block's values
// go through op.out, and every reduction of the scalar solve (scale, the two
// norms, each Newton step's S1, S2) is a round of huge_allreduce.  The Newton
// iteration is the one of group_soc_reg / warp_soc_mem, warm-started from the
// block's previous root; its results, and so the control flow, are identical
// in every CTA.  Each element is then finished with op.fin.
template <class Op, int NACC>
__device__ void huge_block_proj(const Op& op, const ConeTable& T, int h, int cta, int& round, double (&acc)[NACC]) {
  const int64_t st = T.huge_start[h], d = T.huge_len[h];
  const bool rsoc = T.huge_rsoc[h] != 0;
  const int64_t chunk = (d + T.ctaD - 1) / T.ctaD;
  const int64_t lo = (int64_t)cta * chunk, hi = lo + chunk < d ? lo + chunk : d;
  double* u = op.out + st;
  const double* S = T.S ? T.S + st : nullptr;
  const double gw = S ? (rsoc ? sqrt(S[0] * S[1]) : S[0]) : 1.0;
  auto wt = [&](int64_t i) { return (!S || (rsoc && i == 1)) ? 1.0 : gw / S[i]; };
  const double r2 = 0.7071067811865476;
  // values in SOC form (RSOC: rotate the first two), local max |u| and weight flag
  double mx[2] = {0.0, 0.0};
  for (int64_t i = lo + threadIdx.x; i < hi; i += kThreads) {
    double v = op.z(st + i);
    if (rsoc && i < 2) {
      const double z0 = op.z(st), z1 = op.z(st + 1);
      v = (i == 0) ? (z0 + z1) * r2 : (z0 - z1) * r2;
    }
    u[i] = v;
    mx[0] = fmax(mx[0], fabs(v));
    if (i >= 1 && wt(i) != 1.0) mx[1] = 1.0;
  }
  const bool kmax2[2] = {true, true};
  if (!huge_allreduce<2>(T, cta, round, mx, kmax2)) return;
  const double scale = mx[0];
  const bool weighted = mx[1] != 0.0;
  const bool trivial = scale == 0.0 || !isfinite(scale);
  const double sc = trivial ? 1.0 : scale;
  const double t = __ldcg(u) / sc;
  double2* scr = T.huge_scr + T.huge_soff[h];
  const int64_t lo1 = lo > 1 ? lo : 1;
  double nr[2] = {0.0, 0.0};
  for (int64_t i = lo1 + threadIdx.x; i < hi; i += kThreads) {
    const double D = wt(i), xi = __ldcg(u + i) / sc;
    nr[0] += (D * xi) * (D * xi);
    nr[1] += (xi / D) * (xi / D);
    scr[i] = make_double2(D * D * xi * xi, D);  // the Newton rounds read one 16-byte record per element
  }
  const bool ksum2[2] = {false, false};
  if (!huge_allreduce<2>(T, cta, round, nr, ksum2)) return;
  const double nDx = sqrt(nr[0]), nxD = sqrt(nr[1]);
  const bool inside = trivial || nDx <= t;
  const bool polar = !inside && nxD <= -t;
  // the result p_i = f(u_i): inside p = u, polar p = 0, else p_0 = s0, p_i = u_i * mul(i)
  double s0 = 0.0, mu = 0.0, cc = 0.0;
  int mode = inside ? 0 : (polar ? 1 : (weighted ? 3 : 2));
  if (mode == 2) {
    cc = 0.5 * (1.0 + t / nDx);
    s0 = cc * nDx * sc;
  } else if (mode == 3) {
    if (t == 0.0) {
      double a[1] = {0.0};
      for (int64_t i = (lo > 1 ? lo : 1) + threadIdx.x; i < hi; i += kThreads) {
        const double D = wt(i), y0 = (__ldcg(u + i) / sc) / (1.0 + D * D);
        a[0] += (D * y0) * (D * y0);
      }
      const bool ks1[1] = {false};
      if (!huge_allreduce<1>(T, cta, round, a, ks1)) return;
      s0 = sqrt(a[0]) * sc;
      mu = 1.0;
    } else {
      const double s_lo = fmax(t, 0.0);
      double s = s_lo;
      double* ws = T.soc_ws ? T.soc_ws + T.huge_wc[h] : nullptr;
      const double sw = ws ? __ldcg(ws) / sc : __longlong_as_double(0x7ff8000000000000ll);
      bool first = isfinite(sw) && sw > s_lo;
      if (first) s = sw;
      for (int it = 0; it < 200; ++it) {
        double q[2] = {0.0, 0.0};
        // four records per thread in flight (the same per-thread order as one at a time)
        for (int64_t i0 = lo1 + threadIdx.x; i0 < hi; i0 += 4 * kThreads) {
          double2 e[4];
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const int64_t i = i0 + (int64_t)k * kThreads;
            e[k] = i < hi ? __ldcg(scr + i) : make_double2(0.0, 1.0);
          }
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const double c = e[k].x, D = e[k].y;
            if (c == 0.0) continue;
            const double a = 1.0 + D * D;
            const double iu = __drcp_rn(s * a - t * D * D);  // = 1.0 / x, correctly rounded
            q[0] += c * iu * iu;
            q[1] += c * a * iu * iu * iu;
          }
        }
        if (!huge_allreduce<2>(T, cta, round, q, ksum2)) return;
        const double Q = __drcp_rn(sqrt(q[0]));
        const double dQ = Q * Q * Q * q[1];
        const double step = (1.0 - Q) / dQ;
        if (first) {
          first = false;
          if (step < 0.0) {  // warm start above the root
            s = fmax(s + step, s_lo);
            continue;
          }
        }
        if (!(step > 0.0)) break;
        const double sn = s + step;
        if (!(sn > s)) break;
        s = sn;
        if (step <= 1e-17 * s) break;
      }
      mu = 1.0 - t / s;
      s0 = s * sc;
      if (ws && cta == 0 && threadIdx.x == 0) *ws = s * sc;
    }
  }
  auto pval = [&](int64_t i, double ui) {  // the SOC-form result of element i
    if (mode == 0) return ui;
    if (mode == 1) return 0.0;
    if (i == 0) return s0;
    if (mode == 2) return ui * cc;
    const double D = __ldcg(scr + i).y;
    return ui / (1.0 + mu * D * D);
  };
  for (int64_t i = lo + threadIdx.x; i < hi; i += kThreads) {
    double p = pval(i, __ldcg(u + i));
    if (rsoc && i < 2) {  // rotate back (both elements live in CTA 0's slice)
      const double p0 = pval(0, __ldcg(u)), p1 = pval(1, __ldcg(u + 1));
      p = (i == 0) ? (p0 + p1) * r2 : (p0 - p1) * r2;
    }
    op.fin(st + i, op.z(st + i), p, acc);
  }
}

// Ops of the batched solver restrict work to the elements of selected
// instances: live(j) is false for elements that must not be read or written.
template <class Op>
concept MaskedOp = requires(const Op& o) { o.live(int64_t(0)); };

// Generic update + projection.  Op supplies:
//   NACC, kinds[] (ACC_SUM / ACC_MAX), double* out (result / scratch, length T.len),
//   load(): read scalars; z(j): value before projection; fin(j, z, p, acc): consume.
// EXP: compile the exponential-cone path (its root solve sets the register
// budget of the whole kernel; tables without exp cones use EXP = false).
// HUGE: compile part D (tables with huge blocks only: its code raises the
// register count of the whole kernel, 64 -> 80 without EXP).
template <class Op, bool EXP = true, bool HUGE = false>
__global__ void __launch_bounds__(kThreads, HUGE ? 2 : 1) update_project_kernel(Op op, ConeTable T, double* partials,
                                                                 const int32_t* active) {
  if (active && !*active) return;
  op.load();
  double acc[Op::NACC];
#pragma unroll
  for (int k = 0; k < Op::NACC; ++k) acc[k] = 0.0;
  const int b = (int)blockIdx.x - T.ctaD;  // part D (huge blocks) first: the lowest block indices
  const int nblocks = gridDim.x;
  if (HUGE && b < 0) {
    if constexpr (HUGE) {
      int round = 0;
      for (int h = 0; h < T.nhuge; ++h) huge_block_proj<Op, Op::NACC>(op, T, h, (int)blockIdx.x, round, acc);
    }
  } else if (b < T.ctaA && T.act_chunk) {
    // chunks of the elementwise segments, a CTA per chunk
    const int64_t nch = T.act_meta[0];
    for (int64_t q = b; q < nch; q += T.ctaA) {
      const int2 ch = T.act_chunk[q];
      if ((int)threadIdx.x >= ch.y) continue;
      const int64_t j = (int64_t)ch.x + threadIdx.x;
      if constexpr (MaskedOp<Op>) {
        if (!op.live(j)) continue;
      }
      int32_t kind = T.seg_kind[0];
      for (int s = 1; s < T.nseg; ++s)
        if (j >= T.seg_start[s]) kind = T.seg_kind[s];
      double z = op.z(j);
      double p = elem_proj(kind, z, j, T);
      op.fin(j, z, p, acc);
    }
  } else if (b < T.ctaA) {
    const int64_t stride = (int64_t)T.ctaA * kThreads;
    for (int s = 0; s < T.nseg; ++s) {
      const int64_t j0 = T.seg_start[s], j1 = j0 + T.seg_len[s];
      const int32_t kind = T.seg_kind[s];
      for (int64_t j = j0 + (int64_t)b * kThreads + threadIdx.x; j < j1; j += stride) {
        if constexpr (MaskedOp<Op>) {
          if (!op.live(j)) continue;
        }
        double z = op.z(j);
        double p = elem_proj(kind, z, j, T);
        op.fin(j, z, p, acc);
      }
    }
  } else if (b < T.ctaA + T.ctaB) {
    const int lane = threadIdx.x & 31;
    const int64_t wstride = (int64_t)T.ctaB * kWarps;
    const double r2 = 0.7071067811865476;
    int64_t task0[kCls + 1], cls_off[kCls + 1];
    const int64_t* sched = T.act_sched ? T.act_sched : T.sched;
#pragma unroll
    for (int q = 0; q <= kCls; ++q) {
      task0[q] = T.act_sched ? T.act_meta[1 + q] : T.task0[q];
      cls_off[q] = T.act_sched ? T.act_meta[kCls + 2 + q] : T.cls_off[q];
    }
    for (int64_t task = (int64_t)(b - T.ctaA) * kWarps + (threadIdx.x >> 5); task < task0[kCls];
         task += wstride) {
      int c = 0;
#pragma unroll
      for (int q = 1; q < kCls; ++q)
        if (task >= task0[q]) c = q;
      if (c < kCls - 1) {
        // 32 / g blocks of at most 2 g elements, one per lane group, two elements per lane
        const int g = cls_lanes(c);
        const int gl = lane & (g - 1);
        const int64_t idx = cls_off[c] + (task - task0[c]) * (32 / g) + lane / g;
        bool have = idx < cls_off[c + 1];
        int64_t k = 0, st = 0;
        int d = 0;
        bool rsoc = false;
        if (have && T.act_desc) {
          const int4 de = T.act_desc[idx];
          k = de.z;
          st = de.x;
          if constexpr (MaskedOp<Op>) {
            if (!op.mask[de.w]) have = false;  // group-uniform: a block belongs to one instance
          }
          d = have ? (de.y & 0x3fffffff) : 0;
          rsoc = have && (de.y >> 30) != 0;
        } else if (have) {
          k = sched[idx];
          st = T.wc_start[k];
          if constexpr (MaskedOp<Op>) {
            if (!op.live(st)) have = false;  // group-uniform: a block belongs to one instance
          }
          d = have ? T.wc_len[k] : 0;
          rsoc = have && T.wc_kind[k] == PK_RSOC;
        }
        const double* S = (T.S && have) ? T.S + st : nullptr;
        const double num = (S && d > 0) ? (rsoc ? sqrt(S[0] * S[1]) : S[0]) : 1.0;
        double* wsp = (have && T.soc_ws) ? T.soc_ws + k : nullptr;
        const double wsv = (wsp && gl == 0) ? *wsp : __longlong_as_double(0x7ff8000000000000ll);
        double z[kClsEPL], v[kClsEPL], w[kClsEPL];
        bool wne = false;
#pragma unroll
        for (int q = 0; q < kClsEPL; ++q) {
          const int e = gl + g * q;
          z[q] = e < d ? op.z(st + e) : 0.0;
          v[q] = z[q];
          w[q] = (S && e < d && e >= (rsoc ? 2 : 1)) ? num / S[e] : 1.0;
          wne |= w[q] != 1.0;
        }
        // the group is weighted when any of its elements has a weight != 1 (a vote)
        const unsigned gmask = g == 32 ? kFull : ((1u << g) - 1u) << (lane & ~(g - 1));
        const bool weighted = (__ballot_sync(kFull, wne) & gmask) != 0u;
        auto rotate = [&]() {  // RSOC: the first two elements <-> the SOC form (an involution)
          if (g == 1) {
            const double p0 = v[0], q0 = v[1];
            if (rsoc) {
              v[0] = (p0 + q0) * r2;
              v[1] = (p0 - q0) * r2;
            }
          } else {
            const double p0 = __shfl_sync(kFull, v[0], 0, g), q0 = __shfl_sync(kFull, v[0], 1, g);
            if (rsoc && gl == 0) v[0] = (p0 + q0) * r2;
            if (rsoc && gl == 1) v[0] = (p0 - q0) * r2;
          }
        };
        rotate();
        group_soc_multi<kClsEPL>(v, w, d, weighted, g, wsv, wsp);
        rotate();
#pragma unroll
        for (int q = 0; q < kClsEPL; ++q) {
          const int e = gl + g * q;
          if (e < d) op.fin(st + e, z[q], v[q], acc);
        }
      } else {
        // blocks of more than 32 elements: a warp each, values staged in op.out
        int64_t k, st;
        int32_t d;
        bool rsoc;
        if (T.act_desc) {
          const int4 de = T.act_desc[cls_off[c] + (task - task0[c])];
          if constexpr (MaskedOp<Op>) {
            if (!op.mask[de.w]) continue;  // warp-uniform
          }
          k = de.z;
          st = de.x;
          d = de.y & 0x3fffffff;
          rsoc = (de.y >> 30) != 0;
        } else {
          k = sched[cls_off[c] + (task - task0[c])];
          st = T.wc_start[k];
          if constexpr (MaskedOp<Op>) {
            if (!op.live(st)) continue;  // warp-uniform
          }
          d = T.wc_len[k];
          rsoc = T.wc_kind[k] == PK_RSOC;
        }
        const double* S = T.S ? T.S + st : nullptr;
        double* p = op.out + st;
        for (int64_t i = lane; i < d; i += 32) p[i] = op.z(st + i);
        __syncwarp();
        bool weighted = false;
        if (S) {
          double gw = rsoc ? sqrt(S[0] * S[1]) : S[0];
          bool any = false;
          for (int64_t i = (rsoc ? 2 : 1) + lane; i < d; i += 32) any |= (gw / S[i] != 1.0);
          weighted = __any_sync(kFull, any);
        }
        if (rsoc) {
          if (lane == 0) {
            double p0 = p[0], q0 = p[1];
            p[0] = (p0 + q0) * r2;
            p[1] = (p0 - q0) * r2;
          }
          __syncwarp();
          double gw = S ? sqrt(S[0] * S[1]) : 1.0;
          warp_soc_mem(p, d, [&](int64_t i) { return (i == 1 || !S) ? 1.0 : gw / S[i]; }, weighted);
          __syncwarp();
          if (lane == 0) {
            double a0 = p[0], b0 = p[1];
            p[0] = (a0 + b0) * r2;
            p[1] = (a0 - b0) * r2;
          }
        } else {
          warp_soc_mem(p, d, [&](int64_t i) { return S ? S[0] / S[i] : 1.0; }, weighted);
        }
        __syncwarp();
        for (int64_t i = lane; i < d; i += 32) {
          double pi = p[i];
          op.fin(st + i, op.z(st + i), pi, acc);
        }
        __syncwarp();
      }
    }
  } else if constexpr (EXP) {
    const int64_t tstride = (int64_t)T.ctaC * kThreads;
    const int64_t total = T.act_exp ? T.act_meta[2 * kCls + 3] : T.exp_count + T.dexp_count;
    for (int64_t kk = (int64_t)(b - T.ctaA - T.ctaB) * kThreads + threadIdx.x; kk < total; kk += tstride) {
      const int64_t k = T.act_exp ? (int64_t)T.act_exp[kk] : kk;
      const bool first = k < T.exp_count;
      const int64_t j = first ? T.exp_base + 3 * k : T.dexp_base + 3 * (k - T.exp_count);
      if constexpr (MaskedOp<Op>) {
        if (!op.live(j)) continue;
      }
      const int32_t kind = first ? T.exp_kind : T.dexp_kind;
      double z0 = op.z(j), z1 = op.z(j + 1), z2 = op.z(j + 2);
      double r = z0, s = z1, t = z2;
      double S0 = 1.0, S1 = 1.0, S2 = 1.0;
      if (T.S) {
        S0 = T.S[j];
        S1 = T.S[j + 1];
        S2 = T.S[j + 2];
      }
      double* ws = T.rho_ws ? T.rho_ws + k : nullptr;
      if (kind == PK_EXP) proj_exp_scaled_dev(r, s, t, S0, S1, S2, ws);
      else proj_dexp_scaled_dev(r, s, t, S0, S1, S2, ws);
      op.fin(j, z0, r, acc);
      op.fin(j + 1, z1, s, acc);
      op.fin(j + 2, z2, t, acc);
    }
  }
  block_reduce_store<Op::NACC>(acc, Op::kinds(), partials, nblocks);
  if constexpr (Op::kFusedControl) {
    // last CTA to finish runs the attempt's control step (no waiting: the
    // counter tells each CTA whether it is the last one)
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(&op.st->done_ctas, 1u) == (unsigned)nblocks - 1);
    __syncthreads();
    if (last) control_block(op.st, op.ctrl_px, op.ctrl_nbx, partials, nblocks);
  }
}

// Launch update_project_kernel on table T, with the exp path only when T has exp cones.
template <class Op>
inline void launch_update_project(const Op& op, const ConeTable& T, double* partials, const int32_t* active,
                                  cudaStream_t s) {
  const int grid = table_grid(T);
  const bool exp = T.exp_count + T.dexp_count > 0;
  if constexpr (!MaskedOp<Op>) {  // masked (batched) tables never hold huge blocks
    if (T.nhuge > 0) {
      if (exp) update_project_kernel<Op, true, true><<<grid, kThreads, 0, s>>>(op, T, partials, active);
      else update_project_kernel<Op, false, true><<<grid, kThreads, 0, s>>>(op, T, partials, active);
      return;
    }
  }
  if (exp) update_project_kernel<Op, true><<<grid, kThreads, 0, s>>>(op, T, partials, active);
  else update_project_kernel<Op, false><<<grid, kThreads, 0, s>>>(op, T, partials, active);
}

// ---------------------------------------------------------------------------
// Ops
// ---------------------------------------------------------------------------
__device__ __constant__ int32_t kSum1[1] = {ACC_SUM};
__device__ __constant__ int32_t kSum2[2] = {ACC_SUM, ACC_SUM};
__device__ __constant__ int32_t kSum3[3] = {ACC_SUM, ACC_SUM, ACC_SUM};
__device__ __constant__ int32_t kResid7[7] = {ACC_SUM, ACC_MAX, ACC_MAX, ACC_SUM, ACC_MAX, ACC_SUM, ACC_SUM};

// x = P(x_lag + ps (aty - c)); acc: sum (x - x_lag)^2
struct OpPrimalStep {
  static constexpr int NACC = 1;
  static constexpr bool kFusedControl = false;
  __device__ static const int32_t* kinds() { return kSum1; }
  const double* xl;
  const double* aty;
  const double* c;
  double* out;
  const PdhgState* st;
  double ps;
  __device__ void load() { ps = st->ps; }
  __device__ double z(int64_t j) const { return xl[j] + ps * (aty[j] - c[j]); }
  __device__ void fin(int64_t j, double, double p, double* acc) const {
    out[j] = p;
    double d = p - xl[j];
    acc[0] = fma(d, d, acc[0]);
  }
};

// y = P(y_lag - ds (2 gx - gxl - h)); acc: sum (y - y_lag)^2, sum (y - y_lag)(gx - gxl)
struct OpDualStep {
  static constexpr int NACC = 2;
  static constexpr bool kFusedControl = true;
  __device__ static const int32_t* kinds() { return kSum2; }
  const double* yl;
  const double* gx;
  const double* gxl;
  const double* h;
  double* out;
  PdhgState* st;
  double ds;
  const double* ctrl_px;  // partials of the primal step (control step input)
  int ctrl_nbx;
  __device__ void load() { ds = st->ds; }
  __device__ double z(int64_t i) const { return yl[i] - ds * ((2.0 * gx[i] - gxl[i]) - h[i]); }
  __device__ void fin(int64_t i, double, double p, double* acc) const {
    out[i] = p;
    double d = p - yl[i];
    acc[0] = fma(d, d, acc[0]);
    acc[1] = fma(d, gx[i] - gxl[i], acc[1]);
  }
};

// out = P(base + alpha dir); acc: [0] sum (out - base)^2, [1] sum dir*(out - base),
// [2] sum (out - base)*(g1 - g0) when g1 != NULL (restart binary search, Mnorm)
struct OpAxpyProj {
  static constexpr int NACC = 3;
  static constexpr bool kFusedControl = false;
  __device__ static const int32_t* kinds() { return kSum3; }
  const double* base;
  const double* dir;
  double alpha;
  double* out;
  const double* g1;
  const double* g0;
  __device__ void load() {}
  __device__ double z(int64_t j) const { return base[j] + alpha * dir[j]; }
  __device__ void fin(int64_t j, double, double p, double* acc) const {
    out[j] = p;
    double d = p - base[j];
    acc[0] = fma(d, d, acc[0]);
    acc[1] = fma(dir[j], d, acc[1]);
    if (g1) acc[2] = fma(d, g1[j] - g0[j], acc[2]);
  }
};

// Residual of a vector against its projection: z = a*u + b*w - c*q (any of
// u, w, q may be NULL, scaled elementwise by su / sw when given); p = P(z).
// acc: [0] sum (p-z)^2, [1] max |p-z|, [2] max |p|, [3] sum |p|,
//      [4] max |a*u*su|, [5] sum |a*u*su|, [6] box dual objective contribution
struct OpResidual {
  static constexpr int NACC = 7;
  static constexpr bool kFusedControl = false;
  __device__ static const int32_t* kinds() { return kResid7; }
  const double* u;
  const double* su;
  double a;
  const double* w;
  double b;
  const double* q;
  double* out;
  // dual-objective term of the box block: sum bl_fin * max(z, 0) + bu_fin * min(z, 0) over j < nbox
  const double* bl_fin;
  const double* bu_fin;
  int64_t nbox;
  __device__ void load() {}
  __device__ double uterm(int64_t j) const { return u ? a * u[j] * (su ? su[j] : 1.0) : 0.0; }
  __device__ double z(int64_t j) const {
    double v = uterm(j);
    if (w) v += b * w[j];
    if (q) v -= q[j];
    return v;
  }
  __device__ void fin(int64_t j, double z, double p, double* acc) const {
    if (out) out[j] = p;
    double d = p - z;
    acc[0] = fma(d, d, acc[0]);
    acc[1] = fmax(acc[1], fabs(d));
    acc[2] = fmax(acc[2], fabs(p));
    acc[3] += fabs(p);
    double ut = fabs(uterm(j));
    acc[4] = fmax(acc[4], ut);
    acc[5] += ut;
    if (j < nbox) acc[6] += bl_fin[j] * fmax(z, 0.0) + bu_fin[j] * fmin(z, 0.0);
  }
};

// Dot products / norms of up to 4 vectors in one pass (deterministic).
struct DotSpec {
  const double* a[4];
  const double* b[4];   // second operand (DK_DOT: NULL means a itself; DK_DIFF2: required)
  const double* sa[4];  // optional elementwise divisor of a
  int32_t kind[4];      // DotKind
  int32_t count;
  int64_t len;
};

}  // namespace pdcs
