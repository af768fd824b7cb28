// pdcs_bsearch.cuh -- the restart criterion's binary search on the device.
//
// binary_search (rpdhg_alg_gpu_gen.jl, the normalized duality gap of the
// duality-gap restart) evaluates, for trial radii t, the point
//   xs = P_X(px + (t tau / 2) h1),  ys = P_Y(py + (t sigma / 2) h2),
//   h1 = G' py - c,  h2 = h - G px,
// and bisects on  val(t) = |xs - px|^2 / tau - 2 (ys - py)'G (xs - px) + |ys - py|^2 / sigma
// against the radius r.  Host-driven, every evaluation is a device round
// trip; here a CTA runs the whole search of one instance -- the projections
// of the instance's elements and cones, the instance's rows of G, the sums
// and the bisection's branches -- and returns the final radius and the gap.
// Every thread of the CTA keeps the same copy of the scalar state (the sums
// are broadcast), so the branches are CTA-uniform.
#pragma once
#include "pdcs_batch_kernels.cuh"

namespace pdcs {

constexpr int kBsMaxProbes = 512;  // evaluations per search before the host path takes over

struct BsArgs {
  const int32_t* list;      // instances, a CTA each
  RunTable rx, ry;          // element runs per instance
  const int64_t* cones_x;   // per instance [8]: SOC, RSOC warp-cone and exp, dual-exp ordinal ranges
  const int64_t* cones_y;
  ConeTable X, Y;
  CsrDev G, Gt;
  const double* c;
  const double* h;
  double *h1, *h2, *xs, *ys, *gpx, *gxs;  // scratch (global element indices)
  const double* px[2];
  const double* py[2];
  int nsearch;              // 1, or 2: the second search starts from the first one's radius
  const double* prm;        // per instance [r, tau, sigma, t0]
  double* out;              // per instance [probes, t, value_0, value_1, ok]
};

// X side: xs = P(px + a h1); contributions (d = xs - px): d^2, h1 d
struct BsOpX {
  const double* base;
  const double* dir;
  double* out;
  double a;
  __device__ double z(int64_t j) const { return base[j] + a * dir[j]; }
  __device__ void fin(int64_t j, double, double p, double* acc) const {
    out[j] = p;
    const double d = p - base[j];
    acc[0] = fma(d, d, acc[0]);
    acc[1] = fma(dir[j], d, acc[1]);
  }
};

// Y side: ys = P(py + a h2); contributions: d^2, h2 d, d (G xs - G px)
struct BsOpY {
  const double* base;
  const double* dir;
  double* out;
  const double* g1;
  const double* g0;
  double a;
  __device__ double z(int64_t j) const { return base[j] + a * dir[j]; }
  __device__ void fin(int64_t j, double, double p, double* acc) const {
    out[j] = p;
    const double d = p - base[j];
    acc[2] = fma(d, d, acc[2]);
    acc[3] = fma(dir[j], d, acc[3]);
    acc[4] = fma(d, g1[j] - g0[j], acc[4]);
  }
};

// One SOC / RSOC warp cone k by one warp (the lane-group projection with
// g = 32 for blocks of at most 32 elements -- lanes past the block add exact
// zeros to the group sums -- and the memory path for larger blocks).
template <class Op>
__device__ void bs_wcone(const Op& op, const ConeTable& T, int64_t k, int lane, double* acc) {
  const double r2 = 0.7071067811865476;
  const int64_t st = T.wc_start[k];
  const int32_t d = T.wc_len[k];
  const bool rsoc = T.wc_kind[k] == PK_RSOC;
  const double* S = T.S ? T.S + st : nullptr;
  if (d <= 32) {
    const int g = 32, gl = lane;
    const double z = (gl < d) ? op.z(st + gl) : 0.0;
    double v = z;
    double w = 1.0;
    if (S && gl < d) {
      if (rsoc) w = (gl >= 2) ? sqrt(S[0] * S[1]) / S[gl] : 1.0;
      else w = (gl >= 1) ? S[0] / S[gl] : 1.0;
    }
    const bool weighted = grp_max(w != 1.0 ? 1.0 : 0.0, g) != 0.0;
    {
      const double p0 = __shfl_sync(kFull, v, 0), q0 = __shfl_sync(kFull, v, 1);
      if (rsoc && gl == 0) v = (p0 + q0) * r2;
      if (rsoc && gl == 1) v = (p0 - q0) * r2;
    }
    group_soc_reg(v, w, d, weighted, g, T.soc_ws ? T.soc_ws + k : nullptr);
    {
      const double a0 = __shfl_sync(kFull, v, 0), b0 = __shfl_sync(kFull, v, 1);
      if (rsoc && gl == 0) v = (a0 + b0) * r2;
      if (rsoc && gl == 1) v = (a0 - b0) * r2;
    }
    if (gl < d) op.fin(st + gl, z, v, acc);
    return;
  }
  double* p = op.out + st;
  for (int64_t i = lane; i < d; i += 32) p[i] = op.z(st + i);
  __syncwarp();
  bool weighted = false;
  if (S) {
    const double gw = rsoc ? sqrt(S[0] * S[1]) : S[0];
    bool any = false;
    for (int64_t i = (rsoc ? 2 : 1) + lane; i < d; i += 32) any |= (gw / S[i] != 1.0);
    weighted = __any_sync(kFull, any);
  }
  if (rsoc) {
    if (lane == 0) {
      const double p0 = p[0], q0 = p[1];
      p[0] = (p0 + q0) * r2;
      p[1] = (p0 - q0) * r2;
    }
    __syncwarp();
    const double gw = S ? sqrt(S[0] * S[1]) : 1.0;
    warp_soc_mem(p, d, [&](int64_t i) { return (i == 1 || !S) ? 1.0 : gw / S[i]; }, weighted);
    __syncwarp();
    if (lane == 0) {
      const double a0 = p[0], b0 = p[1];
      p[0] = (a0 + b0) * r2;
      p[1] = (a0 - b0) * r2;
    }
  } else {
    warp_soc_mem(p, d, [&](int64_t i) { return S ? S[0] / S[i] : 1.0; }, weighted);
  }
  __syncwarp();
  for (int64_t i = lane; i < d; i += 32) op.fin(st + i, op.z(st + i), p[i], acc);
  __syncwarp();
}

// Project the instance's elements of one side (runs r0 .. r1 - 1 elementwise,
// its warp cones and exp cones) with op; CTA-collective, ends with a barrier.
// Two blocks of at most 32 elements per warp: block ka in lanes 0-15, kb (-1: none) in
// lanes 16-31, two elements per lane (group_soc_multi; the weights and the RSOC
// rotation as in bs_wcone).
template <class Op>
__device__ void bs_wcone_pair(const Op& op, const ConeTable& T, int64_t ka, int64_t kb, int lane, double* acc) {
  constexpr int g = 16;
  const double r2 = 0.7071067811865476;
  const int gl = lane & (g - 1);
  const int64_t k = lane < g ? ka : kb;
  const bool have = k >= 0;
  const int64_t st = have ? T.wc_start[k] : 0;
  const int d = have ? T.wc_len[k] : 0;
  const bool rsoc = have && T.wc_kind[k] == PK_RSOC;
  const double* S = (T.S && have) ? T.S + st : nullptr;
  const double num = S ? (rsoc ? sqrt(S[0] * S[1]) : S[0]) : 1.0;
  double* wsp = (have && T.soc_ws) ? T.soc_ws + k : nullptr;
  const double wsv = (wsp && gl == 0) ? *wsp : __longlong_as_double(0x7ff8000000000000ll);
  double z[2], v[2], w[2];
  bool wne = false;
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int e = gl + g * q;
    z[q] = e < d ? op.z(st + e) : 0.0;
    v[q] = z[q];
    w[q] = (S && e < d && e >= (rsoc ? 2 : 1)) ? num / S[e] : 1.0;
    wne |= w[q] != 1.0;
  }
  const unsigned gmask = 0xffffu << (lane & g);
  const bool weighted = (__ballot_sync(kFull, wne) & gmask) != 0u;
  auto rotate = [&]() {  // RSOC: the first two elements <-> the SOC form (an involution)
    const double p0 = __shfl_sync(kFull, v[0], 0, g), q0 = __shfl_sync(kFull, v[0], 1, g);
    if (rsoc && gl == 0) v[0] = (p0 + q0) * r2;
    if (rsoc && gl == 1) v[0] = (p0 - q0) * r2;
  };
  rotate();
  group_soc_multi<2>(v, w, d, weighted, g, wsv, wsp);
  rotate();
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int e = gl + g * q;
    if (e < d) op.fin(st + e, z[q], v[q], acc);
  }
}

template <class Op>
__device__ void bs_project(const Op& op, const ConeTable& T, const RunTable& R, int r0, int r1, const int64_t* cr,
                           int64_t k, double* acc) {
  for (int q = r0; q < r1; ++q) {
    const int64_t s0 = R.start[k * kMaxRuns + q], L = R.len[k * kMaxRuns + q];
    for (int64_t j = s0 + threadIdx.x; j < s0 + L; j += kThreads) {
      int32_t kind = T.seg_kind[0];
      for (int s = 1; s < T.nseg; ++s)
        if (j >= T.seg_start[s]) kind = T.seg_kind[s];
      const double z = op.z(j);
      op.fin(j, z, elem_proj(kind, z, j, T), acc);
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int part = 0; part < 2; ++part) {  // two blocks per warp when both have at most 32 elements
    const int64_t c1 = cr[2 * part + 1];
    for (int64_t w = cr[2 * part] + 2 * warp; w < c1; w += 2 * kWarps) {
      const bool hb = w + 1 < c1;
      if (T.wc_len[w] <= 32 && (!hb || T.wc_len[w + 1] <= 32)) {
        bs_wcone_pair(op, T, w, hb ? w + 1 : -1, lane, acc);
      } else {
        bs_wcone(op, T, w, lane, acc);
        if (hb) bs_wcone(op, T, w + 1, lane, acc);
      }
    }
  }
  for (int part = 0; part < 2; ++part) {
    for (int64_t e = cr[4 + 2 * part] + threadIdx.x; e < cr[5 + 2 * part]; e += kThreads) {
      const bool first = e < T.exp_count;
      const int64_t j = first ? T.exp_base + 3 * e : T.dexp_base + 3 * (e - T.exp_count);
      const int32_t kind = first ? T.exp_kind : T.dexp_kind;
      const double z0 = op.z(j), z1 = op.z(j + 1), z2 = op.z(j + 2);
      double r = z0, s = z1, t = z2;
      double S0 = 1.0, S1 = 1.0, S2 = 1.0;
      if (T.S) {
        S0 = T.S[j];
        S1 = T.S[j + 1];
        S2 = T.S[j + 2];
      }
      double* ws = T.rho_ws ? T.rho_ws + e : nullptr;
      if (kind == PK_EXP) proj_exp_scaled_dev(r, s, t, S0, S1, S2, ws);
      else proj_dexp_scaled_dev(r, s, t, S0, S1, S2, ws);
      op.fin(j, z0, r, acc);
      op.fin(j + 1, z1, s, acc);
      op.fin(j + 2, z2, t, acc);
    }
  }
  __syncthreads();  // outputs visible to the whole CTA
}

// out[i] = A_i . v (then scaled: a out[i] + b w[i]) for the rows in runs r0 .. r1 - 1 of
// instance k: groups of g lanes per row (about two nonzeros per lane from the rows'
// mean length), so short rows keep the CTA's lanes busy; CTA-collective, ends with a barrier.
__device__ void bs_rows(const CsrDev& A, const RunTable& R, int r0, int r1, int64_t k, const double* v, double* out,
                        double a, double b, const double* w) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t rows = 0, nz = 0;
  for (int q = r0; q < r1; ++q) {
    const int64_t s0 = R.start[k * kMaxRuns + q], L = R.len[k * kMaxRuns + q];
    rows += L;
    if (L) nz += A.rp[s0 + L] - A.rp[s0];
  }
  int g = 1;
  while (g < 32 && 2 * g * rows < nz) g *= 2;
  const int gl = lane & (g - 1), per = 32 / g;
  for (int q = r0; q < r1; ++q) {
    const int64_t s0 = R.start[k * kMaxRuns + q], s1 = s0 + R.len[k * kMaxRuns + q];
    // the loop bound is uniform across the warp (every lane reaches the shuffles)
    for (int64_t ib = s0 + (int64_t)warp * per; ib < s1; ib += (int64_t)kWarps * per) {
      const int64_t i = ib + lane / g;
      const bool valid = i < s1;
      double s = 0.0;
      if (valid)
        for (int32_t e = A.rp[i] + gl; e < A.rp[i + 1]; e += g) s = fma(A.v[e], v[A.ci[e]], s);
      for (int o = g >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o, g);
      if (valid && gl == 0) out[i] = w ? a * s + b * w[i] : s;
    }
  }
  __syncthreads();
}

// CTA-wide sums of acc[0..4], returned to every thread
__device__ void bs_reduce5(double* acc, double (*sh)[kWarps]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int r = 0; r < 5; ++r) {
    double v = acc[r];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
    if (lane == 0) sh[r][warp] = v;
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < 5; ++r) {
    double v = 0.0;
    for (int w = 0; w < kWarps; ++w) v += sh[r][w];
    acc[r] = v;
  }
  __syncthreads();  // sh is reused by the next evaluation
}

__global__ void __launch_bounds__(kThreads) bsearch_kernel(BsArgs A) {
  const int64_t k = A.list[blockIdx.x];
  __shared__ double sh[5][kWarps];
  const double* prm = A.prm + 4 * k;
  const double r = prm[0], ta = prm[1], si = prm[2];
  double t0 = prm[3];
  const int64_t* cx = A.cones_x + 8 * k;
  const int64_t* cy = A.cones_y + 8 * k;
  int probes = 0;
  bool ok = true;
  double values[2] = {0.0, 0.0};
  for (int sidx = 0; sidx < A.nsearch && ok; ++sidx) {
    const double *px = A.px[sidx], *py = A.py[sidx];
    // h1 = G' py - c (x rows of G'), gpx = G px, h2 = h - G px (y rows of G)
    bs_rows(A.Gt, A.rx, 0, kMaxRuns, k, py, A.h1, 1.0, -1.0, A.c);
    bs_rows(A.G, A.ry, 0, kMaxRuns, k, px, A.gpx, 1.0, 0.0, nullptr);
    for (int q = 0; q < kMaxRuns; ++q) {
      const int64_t s0 = A.ry.start[k * kMaxRuns + q], L = A.ry.len[k * kMaxRuns + q];
      for (int64_t i = s0 + threadIdx.x; i < s0 + L; i += kThreads) A.h2[i] = -1.0 * A.gpx[i] + 1.0 * A.h[i];
    }
    __syncthreads();
    double h1dx = 0.0, h2dy = 0.0;
    // one evaluation at t (every thread returns the same value)
    auto approx = [&](double t) -> double {
      ++probes;
      double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
      BsOpX ox{px, A.h1, A.xs, t * ta / 2};
      bs_project(ox, A.X, A.rx, 0, 1, cx, k, acc);
      bs_rows(A.G, A.ry, 0, kMaxRuns, k, A.xs, A.gxs, 1.0, 0.0, nullptr);
      BsOpY oy{py, A.h2, A.ys, A.gxs, A.gpx, t * si / 2};
      bs_project(oy, A.Y, A.ry, 0, 2, cy, k, acc);
      bs_reduce5(acc, sh);
      h1dx = acc[1];
      h2dy = acc[3];
      return acc[0] / ta - 2.0 * acc[4] + acc[2] / si;
    };
    double t = t0, tR = t, tL = 0.0;
    for (int it = 1; it <= 1000 && ok; ++it) {
      double val = approx(t);
      if (val > r && val < r + 1e-6) {
        tR = t;
        tL = fmax(t - 0.01, 0.0);
        val = approx(tL);
        if (val < r) break;
      }
      if (val < r && val > r - 1e-6) {
        tL = t;
        tR = t + 0.01;
        val = approx(tR);
        if (val > r) break;
      }
      if (val > r) break;
      t *= 2;
      if (probes >= kBsMaxProbes) ok = false;
    }
    double tM = 0.5 * (tR + tL);
    while (ok && tR - tL > 1e-6) {
      tM = 0.5 * (tR + tL);
      const double v = approx(tM);
      if (v < r) tL = tM;
      else tR = tM;
      if (probes >= kBsMaxProbes) ok = false;
    }
    t0 = tM;
    values[sidx] = (h1dx + h2dy) / r;
  }
  if (threadIdx.x == 0) {
    double* o = A.out + 5 * k;
    o[0] = (double)probes;
    o[1] = t0;
    o[2] = values[0];
    o[3] = values[1];
    o[4] = ok ? 1.0 : 0.0;
  }
}

}  // namespace pdcs
