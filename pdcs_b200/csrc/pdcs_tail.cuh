// pdcs_tail.cuh -- the last iterating instances of a batch, a CTA each.
//
// Late in a batched solve only a few instances are still iterating, and they
// are the small ones (the slowest instances of uneven batches converge after
// many times the attempts of the rest, and their blocks hold a few hundred
// variables).  There the iteration graph's six kernels per attempt are almost
// pure launch and dependency latency.  tail_attempts_kernel gives every
// iterating instance one CTA that runs its attempts in a loop until the
// instance halts (or the round's attempt budget ends; FP32 deltas move to new
// FP64 anchors every kTailAnchor attempts, as between rounds of graphs): the same phases in the
// same order as the graph -- G' y_lag over the instance's x rows, the primal
// update + projection, G over its y rows, the dual update + projection, the
// per-instance sums and the shared control_step, the reflection -- with
// __syncthreads between phases instead of kernel boundaries.  The ops are the
// graph's (per-element contributions, per-instance step arrays), so the
// arithmetic differs from the graph's only in summation order.
#pragma once
#include "pdcs_bsearch.cuh"
#include "pdcs_fp32.cuh"

namespace pdcs {

// y0[i] = A_i . x0 (and y1 for NV 2 / kPair) for the rows in instance k's runs
// of R: groups of g lanes per row (g a power of two, about two nonzeros per lane
// from the instance's mean row length), so a CTA has up to 256 rows in flight;
// CTA-collective, ends with a barrier.
template <class T, int NV>
__device__ void tail_rows(const CsrT<T>& A, const RunTable& R, int64_t k, const T* x0, const T* x1, T* y0, T* y1) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t rows = 0, nz = 0;
  for (int q = 0; q < kMaxRuns; ++q) {
    const int64_t s0 = R.start[k * kMaxRuns + q], L = R.len[k * kMaxRuns + q];
    rows += L;
    if (L) nz += A.rp[s0 + L] - A.rp[s0];
  }
  int g = 1;
  while (g < 32 && 2 * g * rows < nz) g *= 2;
  const int gl = lane & (g - 1), per = 32 / g;
  for (int q = 0; q < kMaxRuns; ++q) {
    const int64_t s0 = R.start[k * kMaxRuns + q], s1 = s0 + R.len[k * kMaxRuns + q];
    // the loop bound is uniform across the warp (every lane reaches the shuffles)
    for (int64_t ib = s0 + (int64_t)warp * per; ib < s1; ib += (int64_t)kWarps * per) {
      const int64_t i = ib + lane / g;
      const bool valid = i < s1;
      T a0 = T(0), a1 = T(0);
      if (valid) {
        for (int32_t e = A.rp[i] + gl; e < A.rp[i + 1]; e += g) {
          T u0, u1;
          spmv_gather<NV>(x0, x1, A.ci[e], u0, u1);
          a0 = fma(A.v[e], u0, a0);
          if (NV >= 2) a1 = fma(A.v[e], u1, a1);
        }
      }
      for (int o = g >> 1; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(kFull, a0, o, g);
        if (NV >= 2) a1 += __shfl_xor_sync(kFull, a1, o, g);
      }
      if (valid && gl == 0) {
        y0[i] = a0;
        if (NV >= 2) y1[i] = a1;
      }
    }
  }
  __syncthreads();
}

// The operands of one attempt, FP32-bulk (deltas from FP64 anchors) ...
struct TailFP32 {
  CsrT<float> Gt, G;
  OpPrimalStep32B p;
  OpDualStep32B d;
  float2* dxp;
  double* dxm;
  float* dy;
  float* dyl;
  double* dym;
  float* aty;
  float* gx;
  float* gxl;
  __device__ void spmv_t(const RunTable& rx, int64_t k) const { tail_rows<float, 1>(Gt, rx, k, dyl, nullptr, aty, nullptr); }
  __device__ void spmv_g(const RunTable& ry, int64_t k) const {
    tail_rows<float, kPair>(G, ry, k, &dxp->x, nullptr, gx, gxl);
  }
  // re-anchoring (materialize_kernel then anchor_kernel and the anchor products of
  // Solver::anchor, for this instance): FP64 iterates from the deltas, the anchors moved
  // there, qa = G' ya - c, ra = G xa - h in FP64
  CsrDev Gt64, G64;
  double *x, *xl, *xm, *y, *yl, *ym, *xa, *ya, *qa, *ra;
  const double *c, *h;
  static constexpr bool kAnchored = true;
  __device__ void reanchor(const RunTable& rx, const RunTable& ry, int64_t k) const {
    for (int q = 0; q < kMaxRuns; ++q) {
      const int64_t a = rx.start[k * kMaxRuns + q], L = rx.len[k * kMaxRuns + q];
      for (int64_t j = a + threadIdx.x; j < a + L; j += kThreads) {
        const double an = xa[j];
        const float2 p = dxp[j];
        const double v = an + (double)p.x, vl = an + (double)p.y, vm = an + dxm[j];
        x[j] = v;
        xl[j] = vl;
        xm[j] = vm;
        xa[j] = v;
        dxp[j] = make_float2(0.0f, (float)(vl - v));
        dxm[j] = vm - v;
      }
      const int64_t b = ry.start[k * kMaxRuns + q], M = ry.len[k * kMaxRuns + q];
      for (int64_t i = b + threadIdx.x; i < b + M; i += kThreads) {
        const double an = ya[i];
        const double v = an + (double)dy[i], vl = an + (double)dyl[i], vm = an + dym[i];
        y[i] = v;
        yl[i] = vl;
        ym[i] = vm;
        ya[i] = v;
        dy[i] = 0.0f;
        dyl[i] = (float)(vl - v);
        dym[i] = vm - v;
      }
    }
    __syncthreads();
    tail_rows<double, 1>(Gt64, rx, k, ya, nullptr, qa, nullptr);
    tail_rows<double, 1>(G64, ry, k, xa, nullptr, ra, nullptr);
    for (int q = 0; q < kMaxRuns; ++q) {
      const int64_t a = rx.start[k * kMaxRuns + q], L = rx.len[k * kMaxRuns + q];
      for (int64_t j = a + threadIdx.x; j < a + L; j += kThreads) qa[j] = qa[j] - c[j];
      const int64_t b = ry.start[k * kMaxRuns + q], M = ry.len[k * kMaxRuns + q];
      for (int64_t i = b + threadIdx.x; i < b + M; i += kThreads) ra[i] = ra[i] - h[i];
    }
    __syncthreads();
  }
  __device__ void reflect(const PdhgState& s, const RunTable& rx, const RunTable& ry, int64_t k) const {
    for (int q = 0; q < kMaxRuns; ++q) {
      const int64_t a = rx.start[k * kMaxRuns + q], L = rx.len[k * kMaxRuns + q];
      for (int64_t j = a + threadIdx.x; j < a + L; j += kThreads) reflect32_x(s, dxp, dxm, j);
      const int64_t b = ry.start[k * kMaxRuns + q], M = ry.len[k * kMaxRuns + q];
      for (int64_t i = b + threadIdx.x; i < b + M; i += kThreads) reflect32_y(s, dy, dyl, dym, i);
    }
  }
};

// ... and FP64.
struct TailFP64 {
  CsrDev Gt, G;
  OpPrimalStepB p;
  OpDualStepB d;
  double *x, *xl, *xm, *y, *yl, *ym, *aty, *gx, *gxl;
  static constexpr bool kAnchored = false;
  __device__ void reanchor(const RunTable&, const RunTable&, int64_t) const {}
  __device__ void spmv_t(const RunTable& rx, int64_t k) const { tail_rows<double, 1>(Gt, rx, k, yl, nullptr, aty, nullptr); }
  __device__ void spmv_g(const RunTable& ry, int64_t k) const { tail_rows<double, 2>(G, ry, k, x, xl, gx, gxl); }
  __device__ void reflect(const PdhgState& s, const RunTable& rx, const RunTable& ry, int64_t k) const {
    const double tmp = s.refl_tmp, inv = s.refl_inv, e = s.refl_extra, eta = s.refl_eta, cum = s.refl_cum;
    auto one = [&](double* v, double* vl, double* vm, int64_t j) {
      const double cur = v[j];
      const double nv = tmp * ((1.0 + e) * cur - e * vl[j]) + inv * cur;
      vm[j] = (vm[j] * cum + nv * eta) / (cum + eta);
      v[j] = nv;
      vl[j] = nv;
    };
    for (int q = 0; q < kMaxRuns; ++q) {
      const int64_t a = rx.start[k * kMaxRuns + q], L = rx.len[k * kMaxRuns + q];
      for (int64_t j = a + threadIdx.x; j < a + L; j += kThreads) one(x, xl, xm, j);
      const int64_t b = ry.start[k * kMaxRuns + q], M = ry.len[k * kMaxRuns + q];
      for (int64_t i = b + threadIdx.x; i < b + M; i += kThreads) one(y, yl, ym, i);
    }
  }
};

// FP32 deltas are re-anchored every kTailAnchor attempts of a CTA's loop, the
// iteration graph's cadence (a round of graphs, then the host re-anchors)
constexpr int kTailAnchor = 128;

struct TailArgs {
  const int32_t* list;    // iterating instances, a CTA each
  int32_t max_attempts;   // the round's attempt budget
  BatchCtl ctl;           // states, step arrays, live flags, runs, contributions
  ConeTable X, Y;
  const int64_t* cones_x;  // per instance [8]: warp-cone and exp-cone ranges
  const int64_t* cones_y;
};

template <class P>
__global__ void __launch_bounds__(kThreads) tail_attempts_kernel(TailArgs A, P pk) {
  const int64_t k = A.list[blockIdx.x];
  __shared__ PdhgState ss;
  __shared__ double red[3][kWarps];
  const BatchCtl& c = A.ctl;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) ss = c.sts[k];
  __syncthreads();
  const int64_t* cx = A.cones_x + 8 * k;
  const int64_t* cy = A.cones_y + 8 * k;
  double unused[3];
  for (int att = 0; att < A.max_attempts; ++att) {
    if (!ss.active) break;  // CTA-uniform (read after a barrier)
    if (P::kAnchored && att > 0 && att % kTailAnchor == 0) pk.reanchor(c.rx, c.ry, k);
    pk.spmv_t(c.rx, k);
    bs_project(pk.p, A.X, c.rx, 0, 1, cx, k, unused);
    pk.spmv_g(c.ry, k);
    bs_project(pk.d, A.Y, c.ry, 0, 2, cy, k, unused);
    double a = 0.0, b = 0.0, d = 0.0;
    control_sums<kThreads>(c, k, threadIdx.x, a, b, d);
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(kFull, a, o);
      b += __shfl_down_sync(kFull, b, o);
      d += __shfl_down_sync(kFull, d, o);
    }
    if (lane == 0) {
      red[0][warp] = a;
      red[1][warp] = b;
      red[2][warp] = d;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      a = b = d = 0.0;
      for (int w = 0; w < kWarps; ++w) {
        a += red[0][w];
        b += red[1][w];
        d += red[2][w];
      }
      PdhgState s = ss;
      control_step(s, a, b, d);
      ss = s;
      c.ps[k] = s.ps;
      c.ds[k] = s.ds;
      c.live[k] = s.active ? 1 : 0;
    }
    __syncthreads();
    if (ss.do_reflect) {
      pk.reflect(ss, c.rx, c.ry, k);
      __syncthreads();
    }
  }
  if (threadIdx.x == 0) {
    PdhgState s = ss;
    s.do_reflect = 0;  // applied above
    c.sts[k] = s;
  }
}

}  // namespace pdcs
