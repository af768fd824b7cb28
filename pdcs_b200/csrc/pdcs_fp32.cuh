// pdcs_fp32.cuh -- FP32-bulk PDHG attempts with FP64 anchors.
//
// Between two refinements the iterates are stored as FP32 deltas from FP64
// anchors:
//   x = xa + dx,  x_lag = xa + dxl,  x_avg = xa + dxm (dxm in FP64)
// with dx and dxl interleaved in one array of float2 pairs {dx, dxl}, so the
// SpMV of the pair (G dx, G dxl) gathers 8 bytes per nonzero in one load
//   y = ya + dy,  y_lag = ya + dyl,  y_avg = ya + dym
// and the per-anchor products are precomputed in FP64:
//   qa = G' ya - c,   ra = G xa - h.
// One attempt then needs only FP32 SpMVs of the deltas (G and G' stored in
// FP32): G' y_lag - c = qa + G' dyl,  2 G x - G x_lag - h = ra + 2 G dx - G dxl.
// FP32 rounding is relative to the deltas (the distance moved since the
// anchor), not to the iterates.  Projections -- the exponential-cone root
// included -- the eta_bar sums and the averages are FP64.  The deltas are
// folded back into the FP64 iterates (materialize) at every halt of the
// device loop and the anchors move there (anchor) every round of graphs, so
// the exit checks, restarts and KKT reductions run in FP64 on the FP64 matrix.
#pragma once
#include "pdcs_kernels.cuh"

namespace pdcs {

// ---- single instance ----

// x = P(xa + dxl + ps (qa + aty)); dx = x - xa (FP32); acc: sum (dx - dxl)^2
struct OpPrimalStep32 {
  static constexpr int NACC = 1;
  static constexpr bool kFusedControl = false;
  __device__ static const int32_t* kinds() { return kSum1; }
  const double* xa;
  float2* dxp;  // {dx, dxl}
  const double* qa;
  const float* aty;
  double* out;  // FP64 scratch of the large-SOC path
  const PdhgState* st;
  double ps;
  __device__ void load() { ps = st->ps; }
  __device__ double z(int64_t j) const { return xa[j] + (double)dxp[j].y + ps * (qa[j] + (double)aty[j]); }
  __device__ void fin(int64_t j, double, double p, double* acc) const {
    const float d = (float)(p - xa[j]);
    dxp[j].x = d;
    const double s = (double)d - (double)dxp[j].y;
    acc[0] = fma(s, s, acc[0]);
  }
};

// y = P(ya + dyl - ds (ra + 2 gx - gxl)); dy = y - ya (FP32);
// acc: sum (dy - dyl)^2, sum (dy - dyl)(gx - gxl); the last CTA runs the control step
struct OpDualStep32 {
  static constexpr int NACC = 2;
  static constexpr bool kFusedControl = true;
  __device__ static const int32_t* kinds() { return kSum2; }
  const double* ya;
  const float* dyl;
  const double* ra;
  const float* gx;
  const float* gxl;
  float* dy;
  double* out;
  PdhgState* st;
  double ds;
  const double* ctrl_px;
  int ctrl_nbx;
  __device__ void load() { ds = st->ds; }
  __device__ double z(int64_t i) const {
    return ya[i] + (double)dyl[i] - ds * (ra[i] + (2.0 * (double)gx[i] - (double)gxl[i]));
  }
  __device__ void fin(int64_t i, double, double p, double* acc) const {
    const float d = (float)(p - ya[i]);
    dy[i] = d;
    const double s = (double)d - (double)dyl[i];
    acc[0] = fma(s, s, acc[0]);
    acc[1] = fma(s, (double)gx[i] - (double)gxl[i], acc[1]);
  }
};

// ---- batched (per-instance steps, masked, per-element contributions) ----

struct OpPrimalStep32B {
  static constexpr int NACC = 1;
  static constexpr bool kFusedControl = false;
  __device__ static const int32_t* kinds() { return kSum1; }
  const double* xa;
  float2* dxp;  // {dx, dxl}
  const double* qa;
  const float* aty;
  double* out;
  const int32_t* inst;
  const uint8_t* mask;
  const double* ps;
  double* dxsq;
  __device__ void load() {}
  __device__ bool live(int64_t j) const { return mask[inst[j]] != 0; }
  __device__ double z(int64_t j) const {
    return xa[j] + (double)dxp[j].y + ps[inst[j]] * (qa[j] + (double)aty[j]);
  }
  __device__ void fin(int64_t j, double, double p, double*) const {
    const float d = (float)(p - xa[j]);
    dxp[j].x = d;
    const double s = (double)d - (double)dxp[j].y;
    dxsq[j] = s * s;
  }
};

struct OpDualStep32B {
  static constexpr int NACC = 1;
  static constexpr bool kFusedControl = false;
  __device__ static const int32_t* kinds() { return kSum1; }
  const double* ya;
  const float* dyl;
  const double* ra;
  const float* gx;
  const float* gxl;
  float* dy;
  double* out;
  const int32_t* inst;
  const uint8_t* mask;
  const double* ds;
  double* dysq;
  double* dgdy;
  __device__ void load() {}
  __device__ bool live(int64_t i) const { return mask[inst[i]] != 0; }
  __device__ double z(int64_t i) const {
    return ya[i] + (double)dyl[i] - ds[inst[i]] * (ra[i] + (2.0 * (double)gx[i] - (double)gxl[i]));
  }
  __device__ void fin(int64_t i, double, double p, double*) const {
    const float d = (float)(p - ya[i]);
    dy[i] = d;
    const double s = (double)d - (double)dyl[i];
    dysq[i] = s * s;
    dgdy[i] = s * ((double)gx[i] - (double)gxl[i]);
  }
};

// Reflection + averaging on the deltas (the anchor cancels: tmp + inv = 1):
// returns the new delta of both the iterate and its lag.
__device__ __forceinline__ float reflect32_value(const PdhgState& s, float d, float dl, double& dm) {
  const double tmp = s.refl_tmp, inv = s.refl_inv, e = s.refl_extra, eta = s.refl_eta, cum = s.refl_cum;
  const double cur = (double)d;
  const float nv = (float)(tmp * ((1.0 + e) * cur - e * (double)dl) + inv * cur);
  dm = (dm * cum + (double)nv * eta) / (cum + eta);
  return nv;
}
__device__ __forceinline__ void reflect32_x(const PdhgState& s, float2* dxp, double* dxm, int64_t j) {
  const float2 p = dxp[j];
  const float nv = reflect32_value(s, p.x, p.y, dxm[j]);
  dxp[j] = make_float2(nv, nv);
}
__device__ __forceinline__ void reflect32_y(const PdhgState& s, float* dy, float* dyl, double* dym, int64_t i) {
  const float nv = reflect32_value(s, dy[i], dyl[i], dym[i]);
  dy[i] = nv;
  dyl[i] = nv;
}

__global__ void __launch_bounds__(kThreads) reflect32_kernel(const PdhgState* __restrict__ st,
                                                            float2* __restrict__ dxp, double* __restrict__ dxm,
                                                            int64_t n,
                                                            float* __restrict__ dy, float* __restrict__ dyl,
                                                            double* __restrict__ dym, int64_t m) {
  if (!st->do_reflect) return;
  const PdhgState s = *st;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n + m; i += stride) {
    if (i < n) reflect32_x(s, dxp, dxm, i);
    else reflect32_y(s, dy, dyl, dym, i - n);
  }
}

// batch_reflect_kernel on the deltas: the chunks of the iterating instances, a warp per chunk
__global__ void __launch_bounds__(kThreads) batch_reflect32_kernel(const int32_t* __restrict__ live_cur,
                                                                  const PdhgState* __restrict__ sts,
                                                                  float2* __restrict__ dxp,
                                                                  double* __restrict__ dxm, float* __restrict__ dy,
                                                                  float* __restrict__ dyl, double* __restrict__ dym,
                                                                  const int4* __restrict__ rchunk,
                                                                  const int64_t* __restrict__ n_rchunk) {
  if (*live_cur == 0) return;
  const int64_t nch = *n_rchunk;
  const int lane = threadIdx.x & 31;
  const int64_t wstride = ((int64_t)gridDim.x * blockDim.x) >> 5;
  constexpr int R = 4;  // elements per lane with their loads in flight together
  for (int64_t q = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < nch; q += wstride) {
    const int4 ch = rchunk[q];  // {first element, length, 0 = x / 1 = y, instance}
    const PdhgState& st = sts[ch.w];
    if (!st.do_reflect) continue;
    PdhgState s;  // the reflection's scalars only
    s.refl_tmp = st.refl_tmp;
    s.refl_inv = st.refl_inv;
    s.refl_extra = st.refl_extra;
    s.refl_eta = st.refl_eta;
    s.refl_cum = st.refl_cum;
    for (int i0 = lane; i0 < ch.y; i0 += 32 * R) {
      float d[R], dl[R];
      double dm[R];
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int i = i0 + 32 * u;
        if (i >= ch.y) continue;
        const int64_t j = (int64_t)ch.x + i;
        if (ch.z == 0) {
          const float2 p = dxp[j];
          d[u] = p.x;
          dl[u] = p.y;
          dm[u] = dxm[j];
        } else {
          d[u] = dy[j];
          dl[u] = dyl[j];
          dm[u] = dym[j];
        }
      }
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int i = i0 + 32 * u;
        if (i >= ch.y) continue;
        const int64_t j = (int64_t)ch.x + i;
        const float nv = reflect32_value(s, d[u], dl[u], dm[u]);
        if (ch.z == 0) {
          dxp[j] = make_float2(nv, nv);
          dxm[j] = dm[u];
        } else {
          dy[j] = nv;
          dyl[j] = nv;
          dym[j] = dm[u];
        }
      }
    }
  }
}

// anchor: va = v, d = 0, dl = vl - v, dm = vm - v (elements of masked instances; mask NULL = all).
// d and dl are read at stride ds (2: the interleaved {dx, dxl} pairs).
__global__ void anchor_kernel(const double* __restrict__ v, const double* __restrict__ vl,
                              const double* __restrict__ vm, double* __restrict__ va, float* __restrict__ d,
                              float* __restrict__ dl, int ds, double* __restrict__ dm,
                              const int32_t* __restrict__ inst, const uint8_t* __restrict__ mask, int64_t len) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += stride) {
    if (mask && !mask[inst[i]]) continue;
    const double a = v[i];
    va[i] = a;
    d[i * ds] = 0.0f;
    dl[i * ds] = (float)(vl[i] - a);
    dm[i] = vm[i] - a;
  }
}

// materialize: v = va + d, vl = va + dl, vm = va + dm
__global__ void materialize_kernel(double* __restrict__ v, double* __restrict__ vl, double* __restrict__ vm,
                                   const double* __restrict__ va, const float* __restrict__ d,
                                   const float* __restrict__ dl, int ds, const double* __restrict__ dm,
                                   const int32_t* __restrict__ inst, const uint8_t* __restrict__ mask,
                                   int64_t len) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += stride) {
    if (mask && !mask[inst[i]]) continue;
    const double a = va[i];
    v[i] = a + (double)d[i * ds];
    vl[i] = a + (double)dl[i * ds];
    vm[i] = a + dm[i];
  }
}

// out = u - w on the elements of masked instances (mask NULL = all)
__global__ void masked_sub_kernel(double* __restrict__ out, const double* __restrict__ u, const double* __restrict__ w,
                                  const int32_t* __restrict__ inst, const uint8_t* __restrict__ mask, int64_t len) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += stride) {
    if (mask && !mask[inst[i]]) continue;
    out[i] = u[i] - w[i];
  }
}

__global__ void to_float_kernel(float* __restrict__ out, const double* __restrict__ in, int64_t len) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += stride) out[i] = (float)in[i];
}

}  // namespace pdcs
