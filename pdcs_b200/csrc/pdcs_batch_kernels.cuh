// pdcs_batch_kernels.cuh -- kernels of the batched solver.
//
// K independent instances are merged into one block-diagonal program whose
// vectors are ordered by cone type across instances (all box parts, then all
// SOC blocks, ...), so the single-instance cone tables, SpMV and projection
// kernels apply unchanged.  What differs per instance -- step sizes, the
// eta_bar test, restarts, termination -- lives in an array of PdhgState and in
// per-instance scalar arrays indexed through per-element instance ids.
//
// Every kernel here touches only the elements of the instances selected by a
// per-instance mask, so requests of different instances (at different points
// of their own control flow) never disturb each other's data.
//
// Reductions are per instance and deterministic: kernels write per-element
// contributions, and a warp per instance sums its (at most kMaxRuns)
// contiguous runs in a fixed order.
#pragma once
#include "pdcs_kernels.cuh"

namespace pdcs {

// x runs: box, SOC, RSOC, exp, dual-exp; y runs: zero, nonneg, SOC, RSOC, exp, dual-exp
constexpr int kMaxRuns = 6;

struct RunTable {
  const int64_t* start;  // K * kMaxRuns
  const int64_t* len;
};

// x = P(x_lag + ps[k] (aty - c)); contribution (x - x_lag)^2
struct OpPrimalStepB {
  static constexpr int NACC = 1;
  static constexpr bool kFusedControl = false;
  __device__ static const int32_t* kinds() { return kSum1; }
  const double* xl;
  const double* aty;
  const double* c;
  double* out;
  const int32_t* inst;
  const uint8_t* mask;
  const double* ps;
  double* dxsq;
  __device__ void load() {}
  __device__ bool live(int64_t j) const { return mask[inst[j]] != 0; }
  __device__ double z(int64_t j) const { return xl[j] + ps[inst[j]] * (aty[j] - c[j]); }
  __device__ void fin(int64_t j, double, double p, double*) const {
    out[j] = p;
    const double d = p - xl[j];
    dxsq[j] = d * d;
  }
};

// y = P(y_lag - ds[k] (2 gx - gxl - h)); contributions (y - y_lag)^2, (y - y_lag)(gx - gxl)
struct OpDualStepB {
  static constexpr int NACC = 1;
  static constexpr bool kFusedControl = false;
  __device__ static const int32_t* kinds() { return kSum1; }
  const double* yl;
  const double* gx;
  const double* gxl;
  const double* h;
  double* out;
  const int32_t* inst;
  const uint8_t* mask;
  const double* ds;
  double* dysq;
  double* dgdy;
  __device__ void load() {}
  __device__ bool live(int64_t i) const { return mask[inst[i]] != 0; }
  __device__ double z(int64_t i) const { return yl[i] - ds[inst[i]] * ((2.0 * gx[i] - gxl[i]) - h[i]); }
  __device__ void fin(int64_t i, double, double p, double*) const {
    out[i] = p;
    const double d = p - yl[i];
    dysq[i] = d * d;
    dgdy[i] = d * (gx[i] - gxl[i]);
  }
};

// OpAxpyProj with a per-instance step: out = P(base + alpha[k] dir)
struct OpAxpyProjB {
  static constexpr int NACC = 3;
  static constexpr bool kFusedControl = false;
  __device__ static const int32_t* kinds() { return kSum3; }
  const double* base;
  const double* dir;
  const double* alpha;
  double* out;
  const double* g1;
  const double* g0;
  const int32_t* inst;
  __device__ void load() {}
  __device__ double z(int64_t j) const { return base[j] + alpha[inst[j]] * dir[j]; }
  __device__ void fin(int64_t j, double, double p, double* acc) const {
    out[j] = p;
    double d = p - base[j];
    acc[0] = fma(d, d, acc[0]);
    acc[1] = fma(dir[j], d, acc[1]);
    if (g1) acc[2] = fma(d, g1[j] - g0[j], acc[2]);
  }
};

// Adapter: runs a single-instance op on the masked instances and stores each
// element's accumulator values (what the op would add for that element) as
// contributions contrib[r * stride + j], reduced per instance afterwards.
template <class Op>
struct PerElem {
  static constexpr int NACC = 1;
  static constexpr bool kFusedControl = false;
  __device__ static const int32_t* kinds() { return kSum1; }
  Op op;
  double* out;  // the op's output (scratch of the large-SOC path)
  double* contrib;
  int64_t stride;
  const int32_t* inst;
  const uint8_t* mask;
  __device__ void load() { op.load(); }
  __device__ bool live(int64_t j) const { return mask[inst[j]] != 0; }
  __device__ double z(int64_t j) const { return op.z(j); }
  __device__ void fin(int64_t j, double z, double p, double*) const {
    double a[Op::NACC];
#pragma unroll
    for (int r = 0; r < Op::NACC; ++r) a[r] = 0.0;
    op.fin(j, z, p, a);
#pragma unroll
    for (int r = 0; r < Op::NACC; ++r) contrib[r * stride + j] = a[r];
  }
};

// Per-instance reductions.  Kinds 0-3 follow dots_kernel (DOT, MAXABS,
// SUMABS, DIFF2 with the optional divisor sa); SUM / MAX reduce contributions.
enum SegKind : int32_t { SK_DOT = 0, SK_MAXABS = 1, SK_SUMABS = 2, SK_DIFF2 = 3, SK_SUM = 4, SK_MAX = 5 };
constexpr int kSegMax = 8;

struct SegSide {
  const double* a[kSegMax];
  const double* b[kSegMax];
  const double* sa[kSegMax];
  int32_t kind[kSegMax];
  int32_t count;
};

__device__ __forceinline__ void seg_side(const SegSide& sp, RunTable rt, int64_t k, int lane, double* out) {
  double acc[kSegMax];
#pragma unroll
  for (int r = 0; r < kSegMax; ++r) acc[r] = 0.0;
  for (int q = 0; q < kMaxRuns; ++q) {
    const int64_t s0 = rt.start[k * kMaxRuns + q], L = rt.len[k * kMaxRuns + q];
    for (int64_t i = s0 + lane; i < s0 + L; i += 32) {
#pragma unroll
      for (int r = 0; r < kSegMax; ++r) {
        if (r >= sp.count) break;
        double a = sp.a[r][i];
        if (sp.sa[r]) a /= sp.sa[r][i];
        switch (sp.kind[r]) {
          case SK_DOT: acc[r] = fma(a, sp.b[r] ? sp.b[r][i] : a, acc[r]); break;
          case SK_MAXABS: acc[r] = fmax(acc[r], fabs(a)); break;
          case SK_SUMABS: acc[r] += fabs(a); break;
          case SK_DIFF2: { double d = a - sp.b[r][i]; acc[r] = fma(d, d, acc[r]); } break;
          case SK_SUM: acc[r] += a; break;
          default: acc[r] = fmax(acc[r], a); break;
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < kSegMax; ++r) {
    if (r >= sp.count) break;
    const bool mx = sp.kind[r] == SK_MAXABS || sp.kind[r] == SK_MAX;
    double v = acc[r];
    for (int o = 16; o > 0; o >>= 1) {
      const double w = __shfl_down_sync(kFull, v, o);
      v = mx ? fmax(v, w) : v + w;
    }
    if (lane == 0) out[r] = v;
  }
}

// out[k * stride + r]: x-side results r < X.count, then y-side results
__global__ void __launch_bounds__(kThreads) seg_reduce_kernel(int64_t K, const uint8_t* __restrict__ mask,
                                                             RunTable rx, SegSide X, RunTable ry, SegSide Y,
                                                             double* __restrict__ out, int stride) {
  const int lane = threadIdx.x & 31;
  const int64_t wstride = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t k = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < K; k += wstride) {
    if (mask && !mask[k]) continue;
    if (X.count) seg_side(X, rx, k, lane, out + k * stride);
    if (Y.count) seg_side(Y, ry, k, lane, out + k * stride + X.count);
  }
}

// The merged CSR's nonzeros from the instance-concatenated uploads, a warp per
// merged row: local column j of instance k -> its merged position (the last x
// run of k starting at or before j).  err: a column outside its instance.
__global__ void merge_cols_kernel(int64_t M, const int32_t* __restrict__ rp, const int64_t* __restrict__ src,
                                  const int32_t* __restrict__ row_inst, const int32_t* __restrict__ ci_in,
                                  const double* __restrict__ v_in, const int64_t* __restrict__ xrun_start,
                                  const int64_t* __restrict__ xloc, const int64_t* __restrict__ ncol,
                                  int32_t* __restrict__ ci, double* __restrict__ v, int32_t* __restrict__ err) {
  const int lane = threadIdx.x & 31;
  const int64_t wstride = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < M; r += wstride) {
    const int64_t k = row_inst[r];
    const int64_t s0 = src[r], d0 = rp[r], len = rp[r + 1] - rp[r];
    for (int64_t e = lane; e < len; e += 32) {
      const int64_t j = ci_in[s0 + e];
      int64_t c = 0;
      if (j < 0 || j >= ncol[k]) {
        *err = 1;
      } else {
        int t = kMaxRuns - 1;
        while (t > 0 && j < xloc[k * kMaxRuns + t]) --t;
        c = xrun_start[k * kMaxRuns + t] + (j - xloc[k * kMaxRuns + t]);
      }
      ci[d0 + e] = (int32_t)c;
      v[d0 + e] = v_in[s0 + e];
    }
  }
}

// Control of one batched attempt.  live_cur / live_next: the number of live
// instances at the start of this attempt and of the next one (two slots used
// alternately by consecutive attempts of a graph).  The contributions of an
// instance are summed in a fixed order, then the shared control_step runs.
struct BatchCtl {
  PdhgState* sts;
  double* ps;
  double* ds;
  uint8_t* live;
  RunTable rx, ry;
  const double* dxsq;
  const double* dysq;
  const double* dgdy;
  int32_t* live_cur;
  int32_t* live_next;
  uint32_t* done_ctas;
  int32_t* live_accum;
  const int32_t* act_inst;  // instances iterating this round (NULL: all K)
  const int64_t* n_act;
  // fused tile kernels: per-tile partial sums instead of per-element
  // contributions (tpx: |dx|^2 per G' tile; tpy: |dy|^2, dy'(G dx - G dxl) per
  // G tile) and every instance's tile ranges (K + 1 each); NULL: contributions
  const double* tpx = nullptr;
  const double* tpy = nullptr;
  const int64_t* tfx = nullptr;
  const int64_t* tfy = nullptr;
};

// Per-instance sums of the attempt's contributions (a: |dx|^2, b: |dy|^2,
// d: dy'(G dx - G dxl)) over the instance's runs, by G lanes (lane gl of G)
template <int G>
__device__ __forceinline__ void control_sums(const BatchCtl& c, int64_t k, int gl, double& a, double& b, double& d) {
  if (c.tpx) {  // the instance's tiles, in tile order
    for (int64_t t = c.tfx[k] + gl; t < c.tfx[k + 1]; t += G) a += c.tpx[t];
    for (int64_t t = c.tfy[k] + gl; t < c.tfy[k + 1]; t += G) {
      b += c.tpy[2 * t];
      d += c.tpy[2 * t + 1];
    }
    return;
  }
  for (int q = 0; q < kMaxRuns; ++q) {
    const int64_t s0 = c.rx.start[k * kMaxRuns + q], L = c.rx.len[k * kMaxRuns + q];
    for (int64_t i = s0 + gl; i < s0 + L; i += G) a += c.dxsq[i];
    const int64_t t0 = c.ry.start[k * kMaxRuns + q], M = c.ry.len[k * kMaxRuns + q];
    for (int64_t i = t0 + gl; i < t0 + M; i += G) {
      b += c.dysq[i];
      d += c.dgdy[i];
    }
  }
}

__device__ __forceinline__ void control_apply(const BatchCtl& c, int64_t k, double a, double b, double d, int& nlive) {
  PdhgState s = c.sts[k];
  control_step(s, a, b, d);
  c.sts[k] = s;
  c.ps[k] = s.ps;
  c.ds[k] = s.ds;
  c.live[k] = s.active ? 1 : 0;
  nlive += s.active ? 1 : 0;
}

// CTA_INST: a CTA per instance (few iterating instances, some of them large);
// otherwise a warp per instance (the control steps of many instances run side by side).
template <bool CTA_INST>
__global__ void __launch_bounds__(kThreads) batch_control_kernel(int64_t K, BatchCtl c) {
  if (*c.live_cur == 0) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *c.live_next = 0;
    return;
  }
  const int lane = threadIdx.x & 31;
  const int64_t nk = c.act_inst ? *c.n_act : K;
  int nlive = 0;
  if constexpr (CTA_INST) {
    __shared__ double red[3][kWarps];
    for (int64_t kk = blockIdx.x; kk < nk; kk += gridDim.x) {
      const int64_t k = c.act_inst ? (int64_t)c.act_inst[kk] : kk;
      if (!c.live[k]) {  // CTA-uniform; no step ran for this instance: nothing to reflect
        if (threadIdx.x == 0) c.sts[k].do_reflect = 0;
        continue;
      }
      double a = 0.0, b = 0.0, d = 0.0;
      control_sums<kThreads>(c, k, threadIdx.x, a, b, d);
      for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(kFull, a, o);
        b += __shfl_down_sync(kFull, b, o);
        d += __shfl_down_sync(kFull, d, o);
      }
      if (lane == 0) {
        red[0][threadIdx.x >> 5] = a;
        red[1][threadIdx.x >> 5] = b;
        red[2][threadIdx.x >> 5] = d;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        a = b = d = 0.0;
        for (int w = 0; w < kWarps; ++w) {
          a += red[0][w];
          b += red[1][w];
          d += red[2][w];
        }
        control_apply(c, k, a, b, d, nlive);
      }
      __syncthreads();  // red is reused; live[k] was read by every thread before thread 0 wrote it
    }
  } else {
    const int64_t wstride = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t kk = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; kk < nk; kk += wstride) {
      const int64_t k = c.act_inst ? (int64_t)c.act_inst[kk] : kk;
      if (!c.live[k]) {
        if (lane == 0) c.sts[k].do_reflect = 0;
        continue;
      }
      double a = 0.0, b = 0.0, d = 0.0;
      control_sums<32>(c, k, lane, a, b, d);
      for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(kFull, a, o);
        b += __shfl_down_sync(kFull, b, o);
        d += __shfl_down_sync(kFull, d, o);
      }
      if (lane == 0) control_apply(c, k, a, b, d, nlive);
    }
  }
  // count the instances still live; the last CTA publishes the count
  __shared__ int sh[kWarps];
  for (int o = 16; o > 0; o >>= 1) nlive += __shfl_down_sync(kFull, nlive, o);
  if (lane == 0) sh[threadIdx.x >> 5] = nlive;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < kWarps; ++w) t += sh[w];
    atomicAdd(c.live_accum, t);
    __threadfence();
    if (atomicAdd(c.done_ctas, 1u) == gridDim.x - 1) {
      __threadfence();
      *c.live_next = atomicExch(c.live_accum, 0);
      *c.done_ctas = 0;
    }
  }
}

// Reflection + eta-weighted averaging with per-instance coefficients
// (reflect_kernel per instance); runs when the attempt's control step ran.
// Work: the chunks {first element, length <= kThreads, 0 = x / 1 = y, instance}
// of the iterating instances, a warp per chunk.
__global__ void __launch_bounds__(kThreads) batch_reflect_kernel(const int32_t* __restrict__ live_cur,
                                                                const PdhgState* __restrict__ sts,
                                                                double* __restrict__ x, double* __restrict__ xl,
                                                                double* __restrict__ xm, double* __restrict__ y,
                                                                double* __restrict__ yl, double* __restrict__ ym,
                                                                const int4* __restrict__ rchunk,
                                                                const int64_t* __restrict__ n_rchunk) {
  if (*live_cur == 0) return;
  const int64_t nch = *n_rchunk;
  const int lane = threadIdx.x & 31;
  const int64_t wstride = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t q = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < nch; q += wstride) {
    const int4 ch = rchunk[q];  // {first element, length, 0 = x / 1 = y, instance}: a warp per chunk
    const PdhgState& s = sts[ch.w];
    if (!s.do_reflect) continue;
    double* v = ch.z == 0 ? x : y;
    double* vl = ch.z == 0 ? xl : yl;
    double* vm = ch.z == 0 ? xm : ym;
    const double tmp = s.refl_tmp, inv = s.refl_inv, e = s.refl_extra, eta = s.refl_eta, cum = s.refl_cum;
    for (int i = lane; i < ch.y; i += 32) {
      const int64_t j = (int64_t)ch.x + i;
      const double cur = v[j];
      const double nv = tmp * ((1.0 + e) * cur - e * vl[j]) + inv * cur;
      vm[j] = (vm[j] * cum + nv * eta) / (cum + eta);
      v[j] = nv;
      vl[j] = nv;
    }
  }
}

// out = a[k] u + b[k] v on the elements of masked instances (v may be NULL)
__global__ void masked_axpby_kernel(double* __restrict__ out, const double* __restrict__ a,
                                    const double* __restrict__ u, const double* __restrict__ b,
                                    const double* __restrict__ v, const int32_t* __restrict__ inst,
                                    const uint8_t* __restrict__ mask, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int32_t k = inst[i];
    if (!mask[k]) continue;
    out[i] = a[k] * u[i] + (v ? b[k] * v[i] : 0.0);
  }
}

// Active-row compaction of a bin-ordered row list: flag[q] = 1 for rows of
// masked instances (flag[R] = 0 closes the scan).
__global__ void row_flags_kernel(const int4* __restrict__ rows, int64_t R, const uint8_t* __restrict__ mask,
                                 int32_t* __restrict__ flag) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q <= R; q += stride)
    flag[q] = (q < R && mask[rows[q].w]) ? 1 : 0;
}

// out[pos[q]] = rows[q] for flagged rows (pos: exclusive scan of flag, so the
// bins stay contiguous and in order); cbin[b] = pos[full_bin[b]]
__global__ void row_compact_kernel(const int4* __restrict__ rows, int64_t R, const int32_t* __restrict__ flag,
                                   const int32_t* __restrict__ pos, int4* __restrict__ out,
                                   const int64_t* __restrict__ full_bin, int64_t* __restrict__ cbin) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < R; q += stride)
    if (flag[q]) out[pos[q]] = rows[q];
  if (blockIdx.x == 0 && threadIdx.x <= kBins) cbin[threadIdx.x] = pos[full_bin[threadIdx.x]];
}

// unscaled output: out = (pick[k] ? vm : v) / D
__global__ void batch_output_kernel(double* __restrict__ out, const double* __restrict__ v,
                                    const double* __restrict__ vm, const double* __restrict__ D,
                                    const int32_t* __restrict__ inst, const uint8_t* __restrict__ pick, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    out[i] = (pick[inst[i]] ? vm[i] : v[i]) / D[i];
}

}  // namespace pdcs
