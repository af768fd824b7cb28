// pdcs_device.cuh -- device-side cone projections and warp utilities.
//
// Every projection is the Euclidean projection onto a diagonally scaled cone
// S o K (S = cumulative Ruiz/Pock-Chambolle scaling of the block, or 1):
//   SOC:  S o SOC  = {(s, y): ||(S_0 / S_i) y_i|| <= s}     (preprocess.jl:200-207)
//   RSOC: S o RSOC = {2pq >= ||(sqrt(S_0 S_1) / S_i) z_i||^2} (preprocess.jl:213-221)
//   EXP:  S o K_exp,  K_exp = cl{(r, s, t): s > 0, s e^{r/s} <= t}
//   DEXP: S o K_exp^* (dual exponential cone, via Moreau)
// The reference computes the same projections with tolerance-controlled
// bisection (cuda/moderate_block_proj.cu:259-1180, cuda/exp_proj.cu:7-975);
// here each is a bracketed Newton solve of a univariate reformulation that
// runs to machine precision (derivations in the oracle, oracle/pdcs_oracle.cpp).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pdcs {

constexpr unsigned kFull = 0xffffffffu;

enum ProjKind : int32_t {
  PK_FREE = 0,
  PK_ZERO = 1,
  PK_NONNEG = 2,
  PK_BOX = 3,
  PK_SOC = 4,
  PK_RSOC = 5,
  PK_EXP = 6,
  PK_DEXP = 7,
};

__device__ __forceinline__ double warp_sum_bcast(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return __shfl_sync(kFull, v, 0);  // identical value in every lane
}
__device__ __forceinline__ double warp_max_bcast(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, o));
  return __shfl_sync(kFull, v, 0);
}

// ---------------------------------------------------------------------------
// Weighted second-order cone, one warp per block.
// Element i of the block lives in lane (i % 32) at slot (i / 32); for d <= 32
// callers keep it in a register (v), for larger blocks in memory (p).
// Dw(i) is the weight of tail element i (i >= 1); unweighted: Dw = 1.
//
// Newton on Q(s) = (sum_i c_i / (s(1 + D_i^2) - t D_i^2)^2)^(-1/2) = 1 from
// s0 = max(t, 0): Q is concave increasing, so the iterates climb monotonically
// to the root (exact in one step when all D_i are equal).
// ---------------------------------------------------------------------------

// Register path: d <= 32, lane < d holds its element in v; weight w (lane>=1).
__device__ inline void warp_soc_reg(double& v, double w, int d, bool weighted) {
  const int lane = threadIdx.x & 31;
  const bool act = lane < d;
  double scale = warp_max_bcast(act ? fabs(v) : 0.0);
  if (scale == 0.0 || !isfinite(scale)) return;
  double t = __shfl_sync(kFull, v, 0) / scale;
  double xi = (act && lane >= 1) ? v / scale : 0.0;
  double D = (act && lane >= 1) ? w : 1.0;
  double nDx = sqrt(warp_sum_bcast((D * xi) * (D * xi)));
  double nxD = sqrt(warp_sum_bcast((xi / D) * (xi / D)));
  if (nDx <= t) return;
  if (nxD <= -t) {
    if (act) v = 0.0;
    return;
  }
  if (!weighted) {
    double cc = 0.5 * (1.0 + t / nDx);
    if (lane == 0) v = cc * nDx * scale;
    else if (act) v *= cc;
    return;
  }
  double s, mu;
  if (t == 0.0) {
    double yi = xi / (1.0 + D * D);
    s = sqrt(warp_sum_bcast((D * yi) * (D * yi)));
    mu = 1.0;
  } else {
    s = fmax(t, 0.0);
    double c = D * D * xi * xi;
    double a = 1.0 + D * D;
    for (int it = 0; it < 200; ++it) {
      double S1 = 0.0, S2 = 0.0;
      if (c != 0.0) {
        double iu = 1.0 / (s * a - t * D * D);
        S1 = c * iu * iu;
        S2 = c * a * iu * iu * iu;
      }
      S1 = warp_sum_bcast(S1);
      S2 = warp_sum_bcast(S2);
      double Q = 1.0 / sqrt(S1);
      double dQ = Q * Q * Q * S2;
      double step = (1.0 - Q) / dQ;
      if (!(step > 0.0)) break;
      double sn = s + step;
      if (!(sn > s)) break;
      s = sn;
      if (step <= 1e-17 * s) break;
    }
    mu = 1.0 - t / s;
  }
  if (lane == 0) v = s * scale;
  else if (act) v = v / (1.0 + mu * D * D);
}

// ---------------------------------------------------------------------------
// Lane groups: g lanes (g = 1..32, a power of two) per block, 32 / g blocks per
// warp.  Reductions are xor butterflies within the group followed by a
// broadcast from the group's lane 0 (identical values in every lane).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double grp_sum(double v, int g) {
  if (g == 1) return v;
  for (int o = g >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o, g);
  return __shfl_sync(kFull, v, 0, g);
}
__device__ __forceinline__ double grp_max(double v, int g) {
  if (g == 1) return v;
  for (int o = g >> 1; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, o, g));
  return __shfl_sync(kFull, v, 0, g);
}
__device__ __forceinline__ double grp_bcast(double v, int g) { return g == 1 ? v : __shfl_sync(kFull, v, 0, g); }

// warp_soc_reg for a lane group (block of d <= g elements, element i in group
// lane i).  Every lane runs the same shuffles: groups whose block is inside,
// polar, unweighted or converged idle through the remaining Newton steps.
// ws: the block's warm start of the Newton root (s * scale from its previous
// projection, NaN = none; NULL = no warm start).  Q is concave increasing, so
// from a start above the root one Newton step lands at or below it; from
// there the iterates climb monotonically as in warp_soc_reg.
__device__ inline void group_soc_reg_w(double& v, double w, int d, bool weighted, int g, double ws_in, double* ws);
__device__ inline void group_soc_reg(double& v, double w, int d, bool weighted, int g, double* ws) {
  const double nan = __longlong_as_double(0x7ff8000000000000ll);
  group_soc_reg_w(v, w, d, weighted, g, (ws && (threadIdx.x & (g - 1)) == 0) ? *ws : nan, ws);
}
// The same with the warm start already loaded (ws_in: lane 0 of the group's
// value, NaN for none; ws: where to store the new root, NULL for nowhere), so a
// caller can issue that load together with its other loads.
__device__ inline void group_soc_reg_w(double& v, double w, int d, bool weighted, int g, double ws_in, double* ws) {
  const int gl = threadIdx.x & (g - 1);
  const bool act = gl < d;
  const double scale = grp_max(act ? fabs(v) : 0.0, g);
  const bool trivial = scale == 0.0 || !isfinite(scale);
  const double sc = trivial ? 1.0 : scale;
  const double vs = act ? v / sc : 0.0;  // one division per lane: t is lane 0's
  const double t = grp_bcast(vs, g);
  const double xi = gl >= 1 ? vs : 0.0;
  const double D = (act && gl >= 1) ? w : 1.0;
  const double nDx = sqrt(grp_sum((D * xi) * (D * xi), g));
  const double nxD = sqrt(grp_sum((xi / D) * (xi / D), g));
  const bool inside = trivial || nDx <= t;
  const bool polar = !inside && nxD <= -t;
  const bool rest = !inside && !polar;
  const bool zero_t = rest && weighted && t == 0.0;
  const bool newton = rest && weighted && t != 0.0;
  // t == 0: closed form (computed by every lane of a warp in which some group needs it)
  double s_zero = 0.0;
  if (__any_sync(kFull, zero_t)) {
    const double y0 = xi / (1.0 + D * D);
    s_zero = sqrt(grp_sum((D * y0) * (D * y0), g));
  }
  const double c = D * D * xi * xi;
  const double a = 1.0 + D * D;
  const double s_lo = fmax(t, 0.0);
  double s = s_lo;
  double sw = (newton && gl == 0) ? ws_in : __longlong_as_double(0x7ff8000000000000ll);
  sw = grp_bcast(sw, g) / sc;
  bool first = newton && isfinite(sw) && sw > s_lo;
  if (first) s = sw;
  bool done = !newton;
  for (int it = 0; it < 200; ++it) {
    if (!__any_sync(kFull, !done)) break;
    double S1 = 0.0, S2 = 0.0;
    if (!done && c != 0.0) {
      const double iu = __drcp_rn(s * a - t * D * D);  // = 1.0 / x, correctly rounded
      S1 = c * iu * iu;
      S2 = c * a * iu * iu * iu;
    }
    S1 = grp_sum(S1, g);
    S2 = grp_sum(S2, g);
    if (done) continue;
    const double Q = __drcp_rn(sqrt(S1));
    const double dQ = Q * Q * Q * S2;
    const double step = (1.0 - Q) / dQ;
    if (first) {
      first = false;
      if (step < 0.0) {  // warm start above the root
        s = fmax(s + step, s_lo);
        continue;
      }
    }
    if (!(step > 0.0)) {
      done = true;
      continue;
    }
    const double sn = s + step;
    if (!(sn > s)) {
      done = true;
      continue;
    }
    s = sn;
    if (step <= 1e-17 * s) done = true;
  }
  if (inside) return;
  if (polar) {
    if (act) v = 0.0;
    return;
  }
  if (!weighted) {
    const double cc = 0.5 * (1.0 + t / nDx);
    if (gl == 0) v = cc * nDx * sc;
    else if (act) v *= cc;
    return;
  }
  const double sf = zero_t ? s_zero : s;
  const double mu = zero_t ? 1.0 : 1.0 - t / s;
  if (gl == 0) {
    v = sf * sc;
    if (newton && ws) *ws = s * sc;
  } else if (act) {
    v = v / (1.0 + mu * D * D);
  }
}

// The same projection with E elements per lane: block element e lives in group
// lane e % g, slot e / g (g = 1: a whole block of up to E elements in one lane, no
// shuffles).  Every scalar of group_soc_reg_w is formed the same way from per-lane
// sums over the slots followed by the group's butterflies, so a warp projects 32 / g
// blocks at once with fewer lanes idle and fewer shuffles per block.  w holds the
// slots' weights on entry (1 for element 0 and empty slots).
template <int E>
__device__ inline void group_soc_multi(double (&v)[E], double (&w)[E], int d, bool weighted, int g, double ws_in,
                                       double* ws) {
  const int gl = threadIdx.x & (g - 1);
  double amax = 0.0;
#pragma unroll
  for (int q = 0; q < E; ++q)
    if (gl + g * q < d) amax = fmax(amax, fabs(v[q]));
  const double scale = grp_max(amax, g);
  const bool trivial = scale == 0.0 || !isfinite(scale);
  const double sc = trivial ? 1.0 : scale;
  double xi[E];
  double t0 = 0.0, sdx = 0.0, sxd = 0.0;
#pragma unroll
  for (int q = 0; q < E; ++q) {
    const bool act = gl + g * q < d, head = q == 0 && gl == 0;
    const double vs = act ? v[q] / sc : 0.0;
    if (q == 0) t0 = vs;
    xi[q] = head ? 0.0 : vs;
    if (!act || head) w[q] = 1.0;  // w is D from here on
    sdx += (w[q] * xi[q]) * (w[q] * xi[q]);
    sxd += (xi[q] / w[q]) * (xi[q] / w[q]);
  }
  const double t = grp_bcast(t0, g);
  const double nDx = sqrt(grp_sum(sdx, g));
  const double nxD = sqrt(grp_sum(sxd, g));
  const bool inside = trivial || nDx <= t;
  const bool polar = !inside && nxD <= -t;
  const bool rest = !inside && !polar;
  const bool zero_t = rest && weighted && t == 0.0;
  const bool newton = rest && weighted && t != 0.0;
  double s_zero = 0.0;  // t == 0: closed form
  if (__any_sync(kFull, zero_t)) {
    double acc = 0.0;
#pragma unroll
    for (int q = 0; q < E; ++q) {
      const double y0 = xi[q] / (1.0 + w[q] * w[q]);
      acc += (w[q] * y0) * (w[q] * y0);
    }
    s_zero = sqrt(grp_sum(acc, g));
  }
  const double s_lo = fmax(t, 0.0);
  double s = s_lo;
  double sw = (newton && gl == 0) ? ws_in : __longlong_as_double(0x7ff8000000000000ll);
  sw = grp_bcast(sw, g) / sc;
  bool first = newton && isfinite(sw) && sw > s_lo;
  if (first) s = sw;
  bool done = !newton;
  for (int it = 0; it < 200; ++it) {
    if (!__any_sync(kFull, !done)) break;
    double S1 = 0.0, S2 = 0.0;
    if (!done) {
#pragma unroll
      for (int q = 0; q < E; ++q) {
        const double c = w[q] * w[q] * xi[q] * xi[q];
        if (c != 0.0) {
          const double a = 1.0 + w[q] * w[q];
          const double iu = __drcp_rn(s * a - t * w[q] * w[q]);
          S1 += c * iu * iu;
          S2 += c * a * iu * iu * iu;
        }
      }
    }
    S1 = grp_sum(S1, g);
    S2 = grp_sum(S2, g);
    if (done) continue;
    const double Q = __drcp_rn(sqrt(S1));
    const double dQ = Q * Q * Q * S2;
    const double step = (1.0 - Q) / dQ;
    if (first) {
      first = false;
      if (step < 0.0) {  // warm start above the root
        s = fmax(s + step, s_lo);
        continue;
      }
    }
    if (!(step > 0.0)) {
      done = true;
      continue;
    }
    const double sn = s + step;
    if (!(sn > s)) {
      done = true;
      continue;
    }
    s = sn;
    if (step <= 1e-17 * s) done = true;
  }
  if (inside) return;
  if (polar) {
#pragma unroll
    for (int q = 0; q < E; ++q)
      if (gl + g * q < d) v[q] = 0.0;
    return;
  }
  if (!weighted) {
    const double cc = 0.5 * (1.0 + t / nDx);
#pragma unroll
    for (int q = 0; q < E; ++q) {
      if (q == 0 && gl == 0) v[q] = cc * nDx * sc;
      else if (gl + g * q < d) v[q] *= cc;
    }
    return;
  }
  const double sf = zero_t ? s_zero : s;
  const double mu = zero_t ? 1.0 : 1.0 - t / s;
#pragma unroll
  for (int q = 0; q < E; ++q) {
    if (q == 0 && gl == 0) {
      v[q] = sf * sc;
      if (newton && ws) *ws = s * sc;
    } else if (gl + g * q < d) {
      v[q] = v[q] / (1.0 + mu * w[q] * w[q]);
    }
  }
}

// Memory path for any d: block values in p[0..d), weights from wfun(i).
template <class WF>
__device__ inline void warp_soc_mem(double* p, int64_t d, WF wfun, bool weighted) {
  const int lane = threadIdx.x & 31;
  double scale = 0.0;
  for (int64_t i = lane; i < d; i += 32) scale = fmax(scale, fabs(p[i]));
  scale = warp_max_bcast(scale);
  if (scale == 0.0 || !isfinite(scale)) return;
  double t = p[0] / scale;
  double a1 = 0.0, a2 = 0.0;
  for (int64_t i = 1 + lane; i < d; i += 32) {
    double D = weighted ? wfun(i) : 1.0;
    double xi = p[i] / scale;
    a1 += (D * xi) * (D * xi);
    a2 += (xi / D) * (xi / D);
  }
  double nDx = sqrt(warp_sum_bcast(a1)), nxD = sqrt(warp_sum_bcast(a2));
  if (nDx <= t) return;
  __syncwarp();
  if (nxD <= -t) {
    for (int64_t i = lane; i < d; i += 32) p[i] = 0.0;
    return;
  }
  if (!weighted) {
    double cc = 0.5 * (1.0 + t / nDx);
    for (int64_t i = 1 + lane; i < d; i += 32) p[i] *= cc;
    __syncwarp();
    if (lane == 0) p[0] = cc * nDx * scale;
    return;
  }
  double s, mu;
  if (t == 0.0) {
    double acc = 0.0;
    for (int64_t i = 1 + lane; i < d; i += 32) {
      double D = wfun(i);
      double yi = (p[i] / scale) / (1.0 + D * D);
      acc += (D * yi) * (D * yi);
    }
    s = sqrt(warp_sum_bcast(acc));
    mu = 1.0;
  } else {
    s = fmax(t, 0.0);
    for (int it = 0; it < 200; ++it) {
      double S1 = 0.0, S2 = 0.0;
      for (int64_t i = 1 + lane; i < d; i += 32) {
        double D = wfun(i);
        double xi = p[i] / scale;
        double c = D * D * xi * xi;
        if (c == 0.0) continue;
        double a = 1.0 + D * D;
        double iu = 1.0 / (s * a - t * D * D);
        S1 += c * iu * iu;
        S2 += c * a * iu * iu * iu;
      }
      S1 = warp_sum_bcast(S1);
      S2 = warp_sum_bcast(S2);
      double Q = 1.0 / sqrt(S1);
      double dQ = Q * Q * Q * S2;
      double step = (1.0 - Q) / dQ;
      if (!(step > 0.0)) break;
      double sn = s + step;
      if (!(sn > s)) break;
      s = sn;
      if (step <= 1e-17 * s) break;
    }
    mu = 1.0 - t / s;
  }
  __syncwarp();
  for (int64_t i = 1 + lane; i < d; i += 32) {
    double D = wfun(i);
    p[i] = p[i] / (1.0 + mu * D * D);
  }
  __syncwarp();
  if (lane == 0) p[0] = s * scale;
}

// ---------------------------------------------------------------------------
// Exponential cone (thread per cone).  See the derivation in
// oracle/pdcs_oracle.cpp: on the smooth boundary w = sp (dr rho, ds, dt e^rho),
// v - w = lam (1/dr, (1-rho)/ds, -e^{-rho}/dt), and rho is the unique root,
// among the intervals where sp > 0 and lam > 0, of
//   f(rho) = N1 dt e^rho - dr ds N2 e^{-rho}/dt - t Q(rho).
// ---------------------------------------------------------------------------

struct ExpCtx {
  double r, s, t, dr, ds, dt;
  __device__ double Q(double x) const { return ds * ds + dr * dr * x * (x - 1.0); }
  __device__ double N1(double x) const { return dr * r * (x - 1.0) + ds * s; }
  __device__ double N2(double x) const { return ds * r - dr * s * x; }
  // f(x) e^{-|x|} (same sign as f, never overflows) and its derivative, from one
  // exponential: e^{x-|x|} and e^{-x-|x|} are 1 or e^{-2|x|} = (e^{-|x|})^2.
  // also returns the size of the terms of f, the scale of its rounding noise
  __device__ void gd(double x, int zmask, double& g, double& dg, double& mag) const;
  __device__ void gd(double x, int zmask, double& g, double& dg) const {
    double mag;
    gd(x, zmask, g, dg, mag);
  }
  __device__ double fs(double x, int zmask) const {
    double g, dg;
    gd(x, zmask, g, dg);
    return g;
  }
};

// One out-of-line copy: the exponential is the bulk of the code, and the
// exp-cone kernels are otherwise large enough to stall on instruction fetch.
__device__ __noinline__ void ExpCtx::gd(double x, int zmask, double& g, double& dg, double& mag) const {
  const double e3 = exp(-fabs(x));
  const double e3s = e3 * e3;
  const double e1 = x >= 0.0 ? 1.0 : e3s;
  const double e2 = x >= 0.0 ? e3s : 1.0;
  const double n1 = (zmask & 1) ? 0.0 : N1(x);
  const double n2 = (zmask & 2) ? 0.0 : N2(x);
  const double a = n1 * dt * e1, b = dr * ds * n2 * e2 / dt, c = t * Q(x) * e3;
  const double f = a - b - c;
  const double fp = dt * e1 * (dr * r + n1) + (dr * ds / dt) * e2 * (dr * s + n2) - t * dr * dr * (2.0 * x - 1.0) * e3;
  g = f;
  dg = fp - (x >= 0.0 ? f : -f);
  mag = fabs(a) + fabs(b) + fabs(c);
}

__device__ inline bool d_in_kexp(double r, double s, double t) {
  if (s > 0.0) return s * exp(r / s) <= t;
  return (s == 0.0 && r <= 0.0 && t >= 0.0);
}
__device__ inline bool d_in_kexp_dual(double a, double b, double c) {
  if (a < 0.0) return -a * exp(b / a) <= 2.718281828459045 * c;
  return (a == 0.0 && b >= 0.0 && c >= 0.0);
}

// Bracketed safeguarded Newton on one admissible interval (cold start).
__device__ __noinline__ bool exp_root_bracketed(const ExpCtx& C, double lo, double hi, int tlo, int thi, double p,
                                                double sg, double* rho_out) {
  const double eps = 2.220446049250313e-16;
    double a, ga, b, gb;
    if (isinf(lo)) {
      double step = fmax(1.0, fabs(p));
      a = p;
      ga = sg * C.fs(a, 0);
      for (int k = 0; k < 2100 && ga >= 0.0; ++k) {
        a = p - step;
        step *= 2.0;
        ga = sg * C.fs(a, 0);
      }
    } else {
      // An endpoint at a root of N1 (sp = 0: v on the polar's boundary) or N2
      // (lam = 0: v on the cone's boundary) where f vanishes to rounding is the
      // root itself: v lies on a boundary within rounding of the membership
      // tests, and the sign of f there is noise.
      double dg, mag;
      a = lo;
      C.gd(a, tlo & 3, ga, dg, mag);
      ga *= sg;
      if ((tlo & 3) && fabs(ga) <= 16.0 * eps * mag) { *rho_out = a; return true; }
    }
    if (isinf(hi)) {
      double base = fmax(p, a);
      double step = fmax(1.0, fabs(base));
      b = base;
      gb = sg * C.fs(b, 0);
      for (int k = 0; k < 2100 && gb <= 0.0; ++k) {
        b = base + step;
        step *= 2.0;
        gb = sg * C.fs(b, 0);
      }
    } else {
      double dg, mag;
      b = hi;
      C.gd(b, thi & 3, gb, dg, mag);
      gb *= sg;
      if ((thi & 3) && fabs(gb) <= 16.0 * eps * mag) { *rho_out = b; return true; }
    }
    if (!(isfinite(ga) && isfinite(gb))) return false;
    if (!((ga <= 0.0 && gb >= 0.0) || (ga >= 0.0 && gb <= 0.0))) return false;
    if (ga == 0.0) { *rho_out = a; return true; }
    if (gb == 0.0) { *rho_out = b; return true; }
    double L = a, R = b;
    bool inc = ga < 0.0;
    double x = 0.5 * (L + R);
    for (int it = 0; it < 400; ++it) {
      double gx, dgx;
      C.gd(x, 0, gx, dgx);
      gx *= sg;
      if (gx == 0.0) break;
      if ((gx < 0.0) == inc) L = x; else R = x;
      double lo2 = fmin(L, R), hi2 = fmax(L, R);
      if (hi2 - lo2 <= 2.0 * eps * fmax(1.0, fabs(x))) break;
      double xn = x - gx / (sg * dgx);
      if (!(xn > lo2 && xn < hi2) || !isfinite(xn)) xn = 0.5 * (lo2 + hi2);
      if (xn == x) break;
      x = xn;
    }
    *rho_out = x;
    return true;
}

// rho_hint: warm start (the root of the previous projection of this cone, or NaN)
__device__ inline bool exp_root_dev(const ExpCtx& C, double* rho_out, double rho_hint) {
  double bv[4];
  int bt[4];
  int nb = 0;
  auto push = [&](double x, int tg) {
    if (!isfinite(x)) return;
    for (int q = 0; q < nb; ++q)
      if (bv[q] == x) { bt[q] |= tg; return; }
    int k = nb;
    while (k > 0 && bv[k - 1] > x) { bv[k] = bv[k - 1]; bt[k] = bt[k - 1]; --k; }
    bv[k] = x;
    bt[k] = tg;
    ++nb;
  };
  if (C.r != 0.0) push(1.0 - C.ds * C.s / (C.dr * C.r), 1);
  if (C.s != 0.0) push(C.ds * C.r / (C.dr * C.s), 2);
  double ratio = C.ds / C.dr;
  double disc = 1.0 - 4.0 * ratio * ratio;
  if (disc >= 0.0) {
    double sq = sqrt(disc);
    push(0.5 * (1.0 - sq), 4);
    push(0.5 * (1.0 + sq), 4);
  }
  const double kInfD = __longlong_as_double(0x7ff0000000000000LL);
  const double eps = 2.220446049250313e-16;
  for (int j = 0; j <= nb; ++j) {
    double lo = (j == 0) ? -kInfD : bv[j - 1];
    double hi = (j == nb) ? kInfD : bv[j];
    int tlo = (j == 0) ? 0 : bt[j - 1];
    int thi = (j == nb) ? 0 : bt[j];
    double p;
    if (isinf(lo) && isinf(hi)) p = 0.0;
    else if (isinf(lo)) p = hi - fmax(1.0, fabs(hi));
    else if (isinf(hi)) p = lo + fmax(1.0, fabs(lo));
    else p = 0.5 * (lo + hi);
    double Qp = C.Q(p);
    if (!(C.N1(p) * Qp > 0.0 && C.N2(p) * Qp > 0.0)) continue;
    const double sg = Qp > 0.0 ? 1.0 : -1.0;
    // The admissible interval holds exactly one root (the KKT point), so a
    // Newton sequence that stays inside it converges to the projection.
    if (isfinite(rho_hint) && rho_hint > lo && rho_hint < hi) {
      double x = rho_hint;
      bool ok = false;
      for (int it = 0; it < 12; ++it) {
        double g, dg, mag;
        C.gd(x, 0, g, dg, mag);
        if (fabs(g) <= 8.0 * eps * mag) { ok = true; break; }  // at the rounding floor of f
        double xn = x - g / dg;
        if (!(xn > lo && xn < hi) || !isfinite(xn)) break;
        if (fabs(xn - x) <= 4.0 * eps * fmax(1.0, fabs(x))) { x = xn; ok = true; break; }
        x = xn;
      }
      if (ok) { *rho_out = x; return true; }
    }
    if (exp_root_bracketed(C, lo, hi, tlo, thi, p, sg, rho_out)) return true;
    continue;
  }
  return false;
}


// Projection of (r, s, t) onto (dr, ds, dt) o K_exp, in place.
__device__ inline void proj_exp_scaled_dev(double& r, double& s, double& t, double dr, double ds, double dt,
                                           double* rho_ws = nullptr) {
  if (!(isfinite(r) && isfinite(s) && isfinite(t))) return;
  if (d_in_kexp(r / dr, s / ds, t / dt)) return;
  if (d_in_kexp_dual(-dr * r, -ds * s, -dt * t)) {
    r = s = t = 0.0;
    return;
  }
  if (r <= 0.0 && s <= 0.0) {
    s = 0.0;
    t = fmax(t, 0.0);
    return;
  }
  double scale = fmax(fabs(r), fmax(fabs(s), fabs(t)));
  ExpCtx C{r / scale, s / scale, t / scale, dr, ds, dt};
  double rho;
  const double hint = rho_ws ? *rho_ws : __longlong_as_double(0x7ff8000000000000LL);
  if (exp_root_dev(C, &rho, hint)) {
    if (rho_ws) *rho_ws = rho;
    double q = C.Q(rho), n1 = C.N1(rho), n2 = C.N2(rho);
    double c1 = fabs(n1) / (fabs(dr * C.r * rho) + fabs(dr * C.r) + fabs(ds * C.s));
    double c2 = fabs(n2) / (fabs(ds * C.r) + fabs(dr * C.s * rho));
    bool primal = (c1 >= c2);
    if (rho > 700.0) primal = false;
    if (rho < -700.0) primal = true;
    if (primal) {
      double sp = n1 / q;
      r = sp * dr * rho * scale;
      s = sp * ds * scale;
      t = sp * dt * exp(rho) * scale;
    } else {
      double lam = dr * ds * n2 / q;
      double r2 = (C.r - lam / dr) * scale;
      double s2 = (C.s - lam * (1.0 - rho) / ds) * scale;
      double t2 = (C.t + lam * exp(-rho) / dt) * scale;
      r = r2;
      s = s2;
      t = t2;
    }
    return;
  }
  // not reached for finite data: nearest of the face point and the origin
  double fr = fmin(r, 0.0), ft = fmax(t, 0.0);
  double d1 = (fr - r) * (fr - r) + s * s + (ft - t) * (ft - t);
  double d0 = r * r + s * s + t * t;
  if (d1 <= d0) { r = fr; s = 0.0; t = ft; }
  else { r = s = t = 0.0; }
}

// S o K_exp^* via Moreau: P(v) = v + P_{(1/S) o K}(-v).
__device__ inline void proj_dexp_scaled_dev(double& r, double& s, double& t, double Sr, double Ss, double St,
                                            double* rho_ws = nullptr) {
  double a = -r, b = -s, c = -t;
  proj_exp_scaled_dev(a, b, c, 1.0 / Sr, 1.0 / Ss, 1.0 / St, rho_ws);
  r += a;
  s += b;
  t += c;
}

}  // namespace pdcs
