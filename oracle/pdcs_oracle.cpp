// pdcs_oracle.cpp -- CPU FP64 restatement of the PDCS solver path.
//
// TEST INFRASTRUCTURE ONLY: the checker the CUDA product is compared with.
// The product (pdcs_b200/) never links, loads or calls this file.
//
// Each routine cites the reference file:line it restates (paths relative to
// the PDCS project root).  Where the reference's CPU (src/pdcs_cpu) and GPU
// (src/pdcs_gpu) semantics differ, the GPU semantics are the default and the
// CPU ones sit behind oracle_options.cpu_semantics.
//
// Projections are computed to machine precision with bracketed Newton
// iterations on univariate reformulations of the projection KKT systems
// (derivations in the comments); the reference computes the same Euclidean
// projections with tolerance-based bisection, so both agree to its tolerance.

#include "pdcs_oracle.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using Vec = std::vector<double>;
const double kInf = std::numeric_limits<double>::infinity();
const double kPositiveZero = 1e-20;  // PDCS_GPU.jl:27

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Csr {
  int64_t m = 0, n = 0;
  std::vector<int64_t> rp, ci;
  Vec v;
};

Csr transpose(const Csr& A) {
  Csr T;
  T.m = A.n;
  T.n = A.m;
  T.rp.assign(A.n + 1, 0);
  int64_t nnz = A.rp[A.m];
  T.ci.resize(nnz);
  T.v.resize(nnz);
  for (int64_t k = 0; k < nnz; ++k) T.rp[A.ci[k] + 1]++;
  for (int64_t j = 0; j < A.n; ++j) T.rp[j + 1] += T.rp[j];
  std::vector<int64_t> pos(T.rp.begin(), T.rp.end() - 1);
  for (int64_t i = 0; i < A.m; ++i)
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      int64_t q = pos[A.ci[k]]++;
      T.ci[q] = i;
      T.v[q] = A.v[k];
    }
  return T;
}

void spmv(const Csr& A, const double* x, double* y) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < A.m; ++i) {
    double s = 0.0;
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) s += A.v[k] * x[A.ci[k]];
    y[i] = s;
  }
}

double dot(const Vec& a, const Vec& b) {
  double s = 0.0;
  int64_t n = (int64_t)a.size();
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}
double nrm2(const Vec& a) { return std::sqrt(dot(a, a)); }
double nrminf(const Vec& a) {
  double s = 0.0;
  int64_t n = (int64_t)a.size();
#pragma omp parallel for reduction(max : s) schedule(static)
  for (int64_t i = 0; i < n; ++i) s = std::max(s, std::fabs(a[i]));
  return s;
}
double nrm1(const Vec& a) {
  double s = 0.0;
  int64_t n = (int64_t)a.size();
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (int64_t i = 0; i < n; ++i) s += std::fabs(a[i]);
  return s;
}

// ---------------------------------------------------------------------------
// Projections
// ---------------------------------------------------------------------------

// Euclidean projection of v = (t, x) onto {(s, y): ||D o y||_2 <= s} where
// D = Dw[1..d-1] (Dw == nullptr means D = 1).  Restates the cone semantics of
// soc_proj! / soc_proj_diagonal! (src/pdcs_cpu/soc_rsoc_proj.jl:5-19, 229-375,
// src/pdcs_gpu/cuda/moderate_block_proj.cu:259-293, 670-760).
//
// Boundary case: the KKT conditions give y_i = x_i / (1 + mu D_i^2) and
// s = t / (1 - mu) with mu = 1 - t/s, so s solves
//   Q(s) = (sum_i c_i / u_i(s)^2)^(-1/2) = 1,  c_i = D_i^2 x_i^2,
//   u_i(s) = s (1 + D_i^2) - t D_i^2.
// Q is a (-2)-power mean of functions affine in s, hence concave and
// increasing; Newton from the left end (s = max(t, 0), where Q < 1) climbs
// monotonically to the root and is exact when D is constant.
void proj_soc_w(double* v, int64_t d, const double* Dw) {
  if (d <= 0) return;
  if (d == 1) {
    v[0] = std::max(v[0], 0.0);
    return;
  }
  double scale = 0.0;
  for (int64_t i = 0; i < d; ++i) scale = std::max(scale, std::fabs(v[i]));
  if (scale == 0.0 || !std::isfinite(scale)) return;
  double t = v[0] / scale;
  double nDx2 = 0.0, nxD2 = 0.0;
  for (int64_t i = 1; i < d; ++i) {
    double D = Dw ? Dw[i] : 1.0;
    double xi = v[i] / scale;
    nDx2 += (D * xi) * (D * xi);
    nxD2 += (xi / D) * (xi / D);
  }
  double nDx = std::sqrt(nDx2), nxD = std::sqrt(nxD2);
  if (nDx <= t) return;  // inside the cone
  if (nxD <= -t) {       // inside the polar cone
    for (int64_t i = 0; i < d; ++i) v[i] = 0.0;
    return;
  }
  if (!Dw) {  // closed form, soc_proj! (soc_rsoc_proj.jl:5-19)
    double cc = 0.5 * (1.0 + t / nDx);
    v[0] = cc * nDx * scale;
    for (int64_t i = 1; i < d; ++i) v[i] *= cc;
    return;
  }
  double s, mu;
  if (t == 0.0) {
    double acc = 0.0;
    for (int64_t i = 1; i < d; ++i) {
      double D = Dw[i];
      double yi = (v[i] / scale) / (1.0 + D * D);
      acc += (D * yi) * (D * yi);
    }
    s = std::sqrt(acc);
    mu = 1.0;
  } else {
    s = std::max(t, 0.0);
    for (int it = 0; it < 200; ++it) {
      double S1 = 0.0, S2 = 0.0;
      for (int64_t i = 1; i < d; ++i) {
        double D = Dw[i];
        double xi = v[i] / scale;
        double c = D * D * xi * xi;
        if (c == 0.0) continue;
        double a = 1.0 + D * D;
        double u = s * a - t * D * D;
        double iu = 1.0 / u;
        S1 += c * iu * iu;
        S2 += c * a * iu * iu * iu;
      }
      double Q = 1.0 / std::sqrt(S1);
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
  v[0] = s * scale;
  for (int64_t i = 1; i < d; ++i) {
    double D = Dw[i];
    v[i] = v[i] / (1.0 + mu * D * D);
  }
}

// Projection onto S o SOC: weights D_i = S_0 / S_i
// (Dr_product_inv_normalized, src/pdcs_gpu/preprocess.jl:200-207).
void proj_soc_scaled(double* v, int64_t d, const double* S) {
  if (!S) {
    proj_soc_w(v, d, nullptr);
    return;
  }
  thread_local Vec w;
  w.assign(d, 1.0);
  bool all_one = true;
  for (int64_t i = 1; i < d; ++i) {
    w[i] = S[0] / S[i];
    if (w[i] != 1.0) all_one = false;
  }
  proj_soc_w(v, d, all_one ? nullptr : w.data());
}

// Projection onto S o RSOC = {(p, q, z): 2 p q >= ||D o z||^2, p, q >= 0},
// D_i = sqrt(S_0 S_1) / S_i (preprocess.jl:213-221; rsoc_proj! and
// rsoc_proj_diagonal!, soc_rsoc_proj.jl:84-178, 477-822).  The rotation
// a = (p+q)/sqrt2, b = (p-q)/sqrt2 maps it isometrically onto the weighted SOC
// {a >= ||(b, D o z)||}, so the projection is rotate -> proj_soc_w -> rotate back.
void proj_rsoc_scaled(double* v, int64_t d, const double* S) {
  if (d < 3) {  // degenerate: treat as nonnegative orthant on (p, q)
    for (int64_t i = 0; i < d; ++i) v[i] = std::max(v[i], 0.0);
    return;
  }
  const double r2 = std::sqrt(0.5);
  double p = v[0], q = v[1];
  v[0] = (p + q) * r2;
  v[1] = (p - q) * r2;
  thread_local Vec w;
  bool all_one = true;
  if (S) {
    w.assign(d, 1.0);
    double g = std::sqrt(S[0] * S[1]);
    for (int64_t i = 2; i < d; ++i) {
      w[i] = g / S[i];
      if (w[i] != 1.0) all_one = false;
    }
  }
  proj_soc_w(v, d, (S && !all_one) ? w.data() : nullptr);
  double a = v[0], b = v[1];
  v[0] = (a + b) * r2;
  v[1] = (a - b) * r2;
}

bool in_kexp(double r, double s, double t) {
  if (s > 0.0) return s * std::exp(r / s) <= t;
  return (s == 0.0 && r <= 0.0 && t >= 0.0);
}
// K_exp^* = cl{(a, b, c): a < 0, -a e^{b/a} <= e c}
bool in_kexp_dual(double a, double b, double c) {
  if (a < 0.0) return -a * std::exp(b / a) <= std::exp(1.0) * c;
  return (a == 0.0 && b >= 0.0 && c >= 0.0);
}

// Euclidean projection of v = (r, s, t) onto D o K_exp (exponent_proj! and
// exponent_proj_diagonal!, src/pdcs_cpu/exp_proj.jl:653-726; Friberg's
// univariate root-finding form).
//
// On the smooth boundary the projection is w = sp (dr rho, ds, dt e^rho) and
// v - w = lam (1/dr, (1-rho)/ds, -e^{-rho}/dt) with sp, lam > 0 (the two
// directions are orthogonal).  The first two coordinates give, with
//   Q(rho)  = ds^2 + dr^2 rho (rho - 1),
//   N1(rho) = dr r (rho - 1) + ds s,   N2(rho) = ds r - dr s rho,
// sp = N1 / Q and lam = dr ds N2 / Q, and the third coordinate leaves
//   f(rho) = N1 dt e^rho - dr ds N2 e^{-rho} / dt - t Q(rho) = 0
// (the same function as oracle_f_diagonal, exp_proj.jl:30-38, times dr).
// The KKT point is unique, so exactly one root lies where sp > 0 and lam > 0.
// The roots of N1, N2, Q split the real line into at most five intervals on
// each of which those signs are constant; the admissible intervals are
// scanned for a sign change of sign(Q) f and the root is polished by
// bracketed Newton.
struct ExpRootCtx {
  double r, s, t, dr, ds, dt;
  double Q(double x) const { return ds * ds + dr * dr * x * (x - 1.0); }
  double N1(double x) const { return dr * r * (x - 1.0) + ds * s; }
  double N2(double x) const { return ds * r - dr * s * x; }
  // f(x) e^{-|x|}: same sign as f, no overflow for any finite x
  // zero_mask bit 1: x is the root of N1, bit 2: root of N2 (use exact zeros)
  double fs(double x, int zero_mask = 0, double* mag = nullptr) const {
    double ax = std::fabs(x);
    double n1 = (zero_mask & 1) ? 0.0 : N1(x);
    double n2 = (zero_mask & 2) ? 0.0 : N2(x);
    double a = n1 * dt * std::exp(x - ax), b = dr * ds * n2 * std::exp(-x - ax) / dt, c = t * Q(x) * std::exp(-ax);
    if (mag) *mag = std::fabs(a) + std::fabs(b) + std::fabs(c);
    return a - b - c;
  }
  // d/dx [f(x) e^{-|x|}]
  double dfs(double x) const {
    double ax = std::fabs(x), sg = x >= 0.0 ? 1.0 : -1.0;
    double fp = dt * std::exp(x - ax) * (dr * r + N1(x)) + (dr * ds / dt) * std::exp(-x - ax) * (dr * s + N2(x)) -
                t * dr * dr * (2.0 * x - 1.0) * std::exp(-ax);
    return fp - sg * fs(x);
  }
};

bool exp_root(const ExpRootCtx& C, double* rho_out) {
  // breakpoints: roots of N1 (tag 1), N2 (tag 2) and Q (tag 4)
  std::vector<std::pair<double, int>> bt;
  if (C.r != 0.0) bt.push_back({1.0 - C.ds * C.s / (C.dr * C.r), 1});
  if (C.s != 0.0) bt.push_back({C.ds * C.r / (C.dr * C.s), 2});
  double ratio = C.ds / C.dr;
  double disc = 1.0 - 4.0 * ratio * ratio;
  if (disc >= 0.0) {
    double sq = std::sqrt(disc);
    bt.push_back({0.5 * (1.0 - sq), 4});
    bt.push_back({0.5 * (1.0 + sq), 4});
  }
  std::sort(bt.begin(), bt.end());
  std::vector<double> b;
  std::vector<int> tag;
  for (auto& e : bt) {
    if (!std::isfinite(e.first)) continue;
    if (!b.empty() && b.back() == e.first) { tag.back() |= e.second; continue; }
    b.push_back(e.first);
    tag.push_back(e.second);
  }
  size_t K = b.size();
  for (size_t j = 0; j <= K; ++j) {
    double lo = (j == 0) ? -kInf : b[j - 1];
    double hi = (j == K) ? kInf : b[j];
    int tlo = (j == 0) ? 0 : tag[j - 1];
    int thi = (j == K) ? 0 : tag[j];
    double p;
    if (std::isinf(lo) && std::isinf(hi)) p = 0.0;
    else if (std::isinf(lo)) p = hi - std::max(1.0, std::fabs(hi));
    else if (std::isinf(hi)) p = lo + std::max(1.0, std::fabs(lo));
    else p = 0.5 * (lo + hi);
    double Qp = C.Q(p);
    if (!(C.N1(p) * Qp > 0.0 && C.N2(p) * Qp > 0.0)) continue;
    double sg = Qp > 0.0 ? 1.0 : -1.0;
    auto g = [&](double x) { return sg * C.fs(x); };
    double a, ga, bb, gb;
    if (std::isinf(lo)) {  // g -> -inf as x -> -inf on an admissible interval
      double step = std::max(1.0, std::fabs(p));
      a = p;
      ga = g(a);
      for (int k = 0; k < 2100 && ga >= 0.0; ++k) {
        a = p - step;
        step *= 2.0;
        ga = g(a);
      }
    } else {
      // An endpoint at a root of N1 (sp = 0: v on the polar's boundary) or N2
      // (lam = 0: v on the cone's boundary) where f vanishes to rounding is
      // the root itself: v lies on a boundary within rounding of the
      // membership tests above, and the sign of f there is noise.
      double mag;
      a = lo;
      ga = sg * C.fs(a, tlo & 3, &mag);
      if ((tlo & 3) && std::fabs(ga) <= 16.0 * std::numeric_limits<double>::epsilon() * mag) {
        *rho_out = a;
        return true;
      }
    }
    if (std::isinf(hi)) {  // g -> +inf as x -> +inf
      double base = std::max(p, a);
      double step = std::max(1.0, std::fabs(base));
      bb = base;
      gb = g(bb);
      for (int k = 0; k < 2100 && gb <= 0.0; ++k) {
        bb = base + step;
        step *= 2.0;
        gb = g(bb);
      }
    } else {
      double mag;
      bb = hi;
      gb = sg * C.fs(bb, thi & 3, &mag);
      if ((thi & 3) && std::fabs(gb) <= 16.0 * std::numeric_limits<double>::epsilon() * mag) {
        *rho_out = bb;
        return true;
      }
    }
    if (!(std::isfinite(ga) && std::isfinite(gb))) continue;
    if (!((ga <= 0.0 && gb >= 0.0) || (ga >= 0.0 && gb <= 0.0))) continue;
    if (ga == 0.0) { *rho_out = a; return true; }
    if (gb == 0.0) { *rho_out = bb; return true; }
    double L = a, R = bb;
    bool inc = ga < 0.0;
    double x = 0.5 * (L + R);
    for (int it = 0; it < 400; ++it) {
      double gx = g(x);
      if (gx == 0.0) break;
      if ((gx < 0.0) == inc) L = x; else R = x;
      double lo2 = std::min(L, R), hi2 = std::max(L, R);
      if (hi2 - lo2 <= 2.0 * std::numeric_limits<double>::epsilon() * std::max(1.0, std::fabs(x))) break;
      double xn = x - gx / (sg * C.dfs(x));
      if (!(xn > lo2 && xn < hi2) || !std::isfinite(xn)) xn = 0.5 * (lo2 + hi2);
      if (xn == x) break;
      x = xn;
    }
    *rho_out = x;
    return true;
  }
  return false;
}

void proj_exp_scaled_impl(double* v, const double* D) {
  double dr = D ? D[0] : 1.0, ds = D ? D[1] : 1.0, dt = D ? D[2] : 1.0;
  double r = v[0], s = v[1], t = v[2];
  if (!(std::isfinite(r) && std::isfinite(s) && std::isfinite(t))) return;
  if (in_kexp(r / dr, s / ds, t / dt)) return;
  if (in_kexp_dual(-dr * r, -ds * s, -dt * t)) {
    v[0] = v[1] = v[2] = 0.0;
    return;
  }
  if (r <= 0.0 && s <= 0.0) {
    v[0] = r;
    v[1] = 0.0;
    v[2] = std::max(t, 0.0);
    return;
  }
  // homogeneity: solve on v / scale
  double scale = std::max(std::fabs(r), std::max(std::fabs(s), std::fabs(t)));
  ExpRootCtx C{r / scale, s / scale, t / scale, dr, ds, dt};
  double rho;
  if (exp_root(C, &rho)) {
    // Rebuild w from the better-conditioned multiplier: w = sp A(rho) loses
    // accuracy when N1 nearly cancels (sp tiny, e^rho huge), w = v - lam B(rho)
    // when N2 does.
    double q = C.Q(rho), n1 = C.N1(rho), n2 = C.N2(rho);
    double c1 = std::fabs(n1) / (std::fabs(dr * C.r * rho) + std::fabs(dr * C.r) + std::fabs(ds * C.s));
    double c2 = std::fabs(n2) / (std::fabs(ds * C.r) + std::fabs(dr * C.s * rho));
    bool primal = (c1 >= c2);
    if (rho > 700.0) primal = false;
    if (rho < -700.0) primal = true;
    if (primal) {
      double sp = n1 / q;
      v[0] = sp * dr * rho * scale;
      v[1] = sp * ds * scale;
      v[2] = sp * dt * std::exp(rho) * scale;
    } else {
      double lam = dr * ds * n2 / q;
      v[0] = (C.r - lam / dr) * scale;
      v[1] = (C.s - lam * (1.0 - rho) / ds) * scale;
      v[2] = (C.t + lam * std::exp(-rho) / dt) * scale;
    }
    return;
  }
  // fallback (not reached for finite data): best feasible heuristic point
  double cand[2][3] = {{std::min(r, 0.0), 0.0, std::max(t, 0.0)}, {0.0, 0.0, 0.0}};
  double best = kInf;
  int bi = 0;
  for (int k = 0; k < 2; ++k) {
    double dd = (cand[k][0] - r) * (cand[k][0] - r) + (cand[k][1] - s) * (cand[k][1] - s) +
                (cand[k][2] - t) * (cand[k][2] - t);
    if (dd < best) { best = dd; bi = k; }
  }
  v[0] = cand[bi][0];
  v[1] = cand[bi][1];
  v[2] = cand[bi][2];
}

// S o K_exp^*  = {v : v / S in K^*}:  P(v) = v + P_{D K}(-v) with D = 1/S
// (dualExponent_proj_diagonal!, exp_proj.jl:730-739; Moreau decomposition).
void proj_dexp_scaled(double* v, const double* S) {
  double w[3] = {-v[0], -v[1], -v[2]};
  if (S) {
    double D[3] = {1.0 / S[0], 1.0 / S[1], 1.0 / S[2]};
    proj_exp_scaled_impl(w, D);
  } else {
    proj_exp_scaled_impl(w, nullptr);
  }
  v[0] += w[0];
  v[1] += w[1];
  v[2] += w[2];
}

int project_block(int kind, double* v, int64_t len, const double* S, const double* lo,
                  const double* hi) {
  switch (kind) {
    case ORC_FREE: return 0;
    case ORC_ZERO:
      for (int64_t i = 0; i < len; ++i) v[i] = 0.0;
      return 0;
    case ORC_NONNEG:
      for (int64_t i = 0; i < len; ++i) v[i] = std::max(v[i], 0.0);
      return 0;
    case ORC_BOX:
      for (int64_t i = 0; i < len; ++i) v[i] = std::min(std::max(v[i], lo[i]), hi[i]);
      return 0;
    case ORC_SOC: proj_soc_scaled(v, len, S); return 0;
    case ORC_RSOC: proj_rsoc_scaled(v, len, S); return 0;
    case ORC_EXP:
      if (len != 3) return -2;
      proj_exp_scaled_impl(v, S);
      return 0;
    case ORC_DEXP:
      if (len != 3) return -2;
      proj_dexp_scaled(v, S);
      return 0;
  }
  return -1;
}

// ---------------------------------------------------------------------------
// Problem data
// ---------------------------------------------------------------------------

struct Block {
  int kind;
  int64_t start, len;
};

struct Problem {
  int64_t n = 0, m = 0, nb = 0;
  Csr G, Gt;              // scaled operator and its transpose
  Csr Graw, Gtraw;        // original operator (KKT is measured in original scale)
  Vec c, h, bl, bu;       // scaled
  Vec craw, hraw, blraw, buraw, bl_fin, bu_fin, lam_l, lam_u;
  Vec Dr, Dl;             // cumulative scaling (Dr_product, Dl_product)
  double hNrm1 = 0, hNrm2 = 0, hNrmInf = 0, cNrm1 = 0, cNrm2 = 0, cNrmInf = 0;
  std::vector<Block> xb;  // iteration projection of x (S = Dr)
  std::vector<Block> yb;  // iteration projection of y (S = Dl)
  std::vector<Block> conb;   // projection of Gx - h onto K_d (original scale)
  std::vector<Block> slackb; // projection of lambda onto Lambda x K_p^* (original scale)
};

// Ruiz l_inf (src/pdcs_gpu/preprocess.jl:521-591) and Pock-Chambolle
// (preprocess.jl:424-470) equilibration, applied through scale_data!
// (preprocess.jl:300-345): c /= Dr, [bl, bu] *= Dr, G_ij /= (Dl_i Dr_j), h /= Dl.
void scale_data(Problem& P, const Vec& var, const Vec& con) {
  for (int64_t j = 0; j < P.n; ++j) {
    P.c[j] /= var[j];
    P.Dr[j] *= var[j];
  }
  for (int64_t j = 0; j < P.nb; ++j) {
    P.bl[j] *= var[j];
    P.bu[j] *= var[j];
  }
  for (int64_t i = 0; i < P.m; ++i) {
    P.h[i] /= con[i];
    P.Dl[i] *= con[i];
    for (int64_t k = P.G.rp[i]; k < P.G.rp[i + 1]; ++k) P.G.v[k] /= (con[i] * var[P.G.ci[k]]);
  }
}

void precondition(Problem& P, int rescaling) {
  P.Dr.assign(P.n, 1.0);
  P.Dl.assign(P.m, 1.0);
  if (rescaling == 1 || rescaling == 3) {
    for (int it = 0; it < 10; ++it) {
      Vec var(P.n, 0.0), con(P.m, 0.0);
      for (int64_t i = 0; i < P.m; ++i)
        for (int64_t k = P.G.rp[i]; k < P.G.rp[i + 1]; ++k) {
          double a = std::fabs(P.G.v[k]);
          con[i] = std::max(con[i], a);
          var[P.G.ci[k]] = std::max(var[P.G.ci[k]], a);
        }
      for (auto& x : var) x = (x == 0.0) ? 1.0 : std::sqrt(x);
      for (auto& x : con) x = (x == 0.0) ? 1.0 : std::sqrt(x);
      scale_data(P, var, con);
    }
  }
  if (rescaling == 2 || rescaling == 3) {
    // alpha = 1: column sums of |G|^(2-alpha), row sums of |G|^alpha
    Vec var(P.n, 0.0), con(P.m, 0.0);
    for (int64_t i = 0; i < P.m; ++i)
      for (int64_t k = P.G.rp[i]; k < P.G.rp[i + 1]; ++k) {
        double a = std::fabs(P.G.v[k]);
        con[i] += a;
        var[P.G.ci[k]] += a;
      }
    for (auto& x : var) x = (x == 0.0) ? 1.0 : std::sqrt(x);
    for (auto& x : con) x = (x == 0.0) ? 1.0 : std::sqrt(x);
    scale_data(P, var, con);
  }
}

int build_problem(const oracle_problem* p, int rescaling, Problem& P) {
  P.n = p->n;
  P.m = p->m;
  P.nb = p->nb;
  int64_t msum = p->mGzero + p->mGnonneg + 3 * (p->expG + p->dual_expG);
  for (int64_t i = 0; i < p->n_socG; ++i) msum += p->socG[i];
  for (int64_t i = 0; i < p->n_rsocG; ++i) msum += p->rsocG[i];
  if (msum != p->m) return -3;  // rpdhg_alg_gpu_gen.jl:1334-1336
  for (int64_t i = 0; i < p->n_socG; ++i) if (p->socG[i] < 2) return -4;   // :84
  for (int64_t i = 0; i < p->n_rsocG; ++i) if (p->rsocG[i] < 3) return -5; // :94
  for (int64_t i = 0; i < p->n_soc_x; ++i) if (p->soc_x[i] < 2) return -4;
  for (int64_t i = 0; i < p->n_rsoc_x; ++i) if (p->rsoc_x[i] < 3) return -5;
  for (int64_t j = 0; j < p->nb; ++j) if (!(p->bl[j] <= p->bu[j])) return -6;  // :1374
  int64_t nsum = p->nb + 3 * (p->exp_x + p->dual_exp_x);
  for (int64_t i = 0; i < p->n_soc_x; ++i) nsum += p->soc_x[i];
  for (int64_t i = 0; i < p->n_rsoc_x; ++i) nsum += p->rsoc_x[i];
  if (nsum > p->n) return -7;
  P.Graw.m = p->m;
  P.Graw.n = p->n;
  P.Graw.rp.assign(p->rowptr, p->rowptr + p->m + 1);
  P.Graw.ci.assign(p->colind, p->colind + p->nnz);
  P.Graw.v.assign(p->val, p->val + p->nnz);
  P.Gtraw = transpose(P.Graw);
  P.G = P.Graw;
  P.craw.assign(p->c, p->c + p->n);
  P.hraw.assign(p->h, p->h + p->m);
  P.blraw.assign(p->bl, p->bl + p->nb);
  P.buraw.assign(p->bu, p->bu + p->nb);
  P.c = P.craw;
  P.h = P.hraw;
  P.bl = P.blraw;
  P.bu = P.buraw;
  P.bl_fin = P.blraw;
  P.bu_fin = P.buraw;
  P.lam_l.resize(p->nb);
  P.lam_u.resize(p->nb);
  for (int64_t j = 0; j < p->nb; ++j) {
    if (std::isinf(P.bl_fin[j])) P.bl_fin[j] = 0.0;
    if (std::isinf(P.bu_fin[j])) P.bu_fin[j] = 0.0;
    // gen_lambd (src/pdcs_gpu/def_rpdhg_gen.jl:5-17)
    P.lam_l[j] = (P.buraw[j] == kInf) ? 0.0 : -kInf;
    P.lam_u[j] = (P.blraw[j] == -kInf) ? 0.0 : kInf;
  }
  // cal_constant on the raw data (def_struct.jl:968-976)
  P.hNrm1 = nrm1(P.hraw);
  P.hNrm2 = nrm2(P.hraw);
  P.hNrmInf = nrminf(P.hraw);
  P.cNrm1 = nrm1(P.craw);
  P.cNrm2 = nrm2(P.craw);
  P.cNrmInf = nrminf(P.craw);
  precondition(P, rescaling);
  P.Gt = transpose(P.G);

  // block tables (rpdhg_alg_gpu_gen.jl:60-120; codes def_rpdhg_gen.jl:265-279, 598-616)
  int64_t s = 0;
  if (p->nb > 0) {
    P.xb.push_back({ORC_BOX, 0, p->nb});
    P.slackb.push_back({ORC_BOX, 0, p->nb});
  }
  s = p->nb;
  for (int64_t i = 0; i < p->n_soc_x; ++i) {
    P.xb.push_back({ORC_SOC, s, p->soc_x[i]});
    P.slackb.push_back({ORC_SOC, s, p->soc_x[i]});
    s += p->soc_x[i];
  }
  for (int64_t i = 0; i < p->n_rsoc_x; ++i) {
    P.xb.push_back({ORC_RSOC, s, p->rsoc_x[i]});
    P.slackb.push_back({ORC_RSOC, s, p->rsoc_x[i]});
    s += p->rsoc_x[i];
  }
  for (int64_t i = 0; i < p->exp_x; ++i) {
    P.xb.push_back({ORC_EXP, s, 3});       // code 27
    P.slackb.push_back({ORC_DEXP, s, 3});  // code 28
    s += 3;
  }
  for (int64_t i = 0; i < p->dual_exp_x; ++i) {
    P.xb.push_back({ORC_DEXP, s, 3});      // code 29
    P.slackb.push_back({ORC_EXP, s, 3});   // code 26
    s += 3;
  }
  s = 0;
  if (p->mGzero > 0) {
    P.yb.push_back({ORC_FREE, 0, p->mGzero});    // code 1
    P.conb.push_back({ORC_ZERO, 0, p->mGzero});  // code 2
  }
  s = p->mGzero;
  if (p->mGnonneg > 0) {
    P.yb.push_back({ORC_NONNEG, s, p->mGnonneg});
    P.conb.push_back({ORC_NONNEG, s, p->mGnonneg});
  }
  s += p->mGnonneg;
  for (int64_t i = 0; i < p->n_socG; ++i) {
    P.yb.push_back({ORC_SOC, s, p->socG[i]});
    P.conb.push_back({ORC_SOC, s, p->socG[i]});
    s += p->socG[i];
  }
  for (int64_t i = 0; i < p->n_rsocG; ++i) {
    P.yb.push_back({ORC_RSOC, s, p->rsocG[i]});
    P.conb.push_back({ORC_RSOC, s, p->rsocG[i]});
    s += p->rsocG[i];
  }
  for (int64_t i = 0; i < p->expG; ++i) {
    P.yb.push_back({ORC_DEXP, s, 3});   // code 12: y in Dl o K_exp^*
    P.conb.push_back({ORC_EXP, s, 3});  // code 13
    s += 3;
  }
  for (int64_t i = 0; i < p->dual_expG; ++i) {
    P.yb.push_back({ORC_EXP, s, 3});     // code 15: y in Dl o K_exp
    P.conb.push_back({ORC_DEXP, s, 3});  // code 16
    s += 3;
  }
  return 0;
}

void project_all(const std::vector<Block>& B, double* v, const double* S, const double* lo,
                 const double* hi) {
  int64_t nb = (int64_t)B.size();
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t b = 0; b < nb; ++b) {
    const Block& k = B[b];
    project_block(k.kind, v + k.start, k.len, S ? S + k.start : nullptr, lo ? lo + k.start : nullptr,
                  hi ? hi + k.start : nullptr);
  }
}

// ---------------------------------------------------------------------------
// Solver state
// ---------------------------------------------------------------------------

struct Converge {
  double pobj = 1e30, dobj = 1e30, abs_gap = 1e30, rel_gap = 1e30;
  double linf_rel_p = 1e30, linf_rel_d = 1e30, l2_rel_p = 1e30, l2_rel_d = 1e30;
  double linf_abs_p = 1e30, linf_abs_d = 1e30, l2_abs_p = 1e30, l2_abs_d = 1e30;
  int status = 7;  // 7 continue, 0 optimal, 8 nan, 9 inf
};

struct Infea {
  double max_primal_ray_inf = 1e30, primal_ray_obj = 1e30, max_dual_ray_inf = 1e30, dual_ray_obj = 1e30;
  double primal_ray_norm = 0, dual_ray_norm = 0;
  std::vector<double> ptrend, dtrend;  // circular buffers of length 20
  int status = 7;
};

struct Solver {
  Problem P;
  oracle_options o;
  int64_t n = 0, m = 0;
  Vec x, xl, xm, y, yl, ym;       // current, lag, mean (scaled space)
  Vec x0, y0, x0l, y0l;           // restart anchors
  Vec xbest, ybest;
  Vec tn1, tn2, tn3, tm1, tm2, tm3;  // temporaries
  double tau = 0.9, sigma = 0.9, omega = 1.0;
  double proj_abs_tol = 1e-11, proj_rel_tol = 1e-11, proj_base_tol = 1e-9;
  double beta_suff = 0.4, beta_nec = 0.8, beta_suff_kkt = 0.4, beta_nec_kkt = 0.8, beta_art = 0.223;
  int64_t iter = 0, iter_stepsize = 0, restart_used = 0, trig_mean = 0, trig_ergodic = 0;
  double ndg[2] = {1e30, 1e30}, ndg_thr = 0, ndg_r = 1e30, kkt_err[2] = {1e30, 1e30}, kkt_thr = 0;
  bool dgap_flag = true;
  double bs_t0 = 1.0, max_kkt = 1e30, min_kkt = 1e30;
  double pres_best = 1e30, dres_best = 1e30;
  Converge ci[2];
  Infea ii[2];
  int exit_code = 7;
  double pobj = 1e30, dobj = 1e30;
  double t_start = 0;
  int returned_seq = 0;
  int64_t check_count = 0;
  bool attempt_limit_hit = false;

  double decay() const { return std::min(0.9 + 0.1 * std::log10(max_kkt * 1e5), 1.0); }

  void proj_x(double* v) { project_all(P.xb, v, P.Dr.data(), P.bl.data(), P.bu.data()); }
  void proj_y(double* v) { project_all(P.yb, v, P.Dl.data(), nullptr, nullptr); }

  // Mnorm (rpdhg_alg_gpu_gen.jl:133-138): x'x/tau - 2 y'Gx + y'y/sigma
  double mnorm(const Vec& dx, const Vec& dy, double ta, double si) {
    spmv(P.G, dx.data(), tm3.data());
    return dot(dx, dx) / ta - 2.0 * dot(dy, tm3) + dot(dy, dy) / si;
  }

  // converge_info_calculation_diagonal! (rpdhg_alg_gpu_gen_scaling.jl:126-183);
  // cpu_semantics switches to rpdhg_alg_cpu_gen_scaling.jl:84-131.
  void converge_info(const Vec& xr, const Vec& yr, Converge& C) {
    Vec aty(n), lam(n), pl(n), gx(m), r(m), pr(m);
    double pobj_ = dot(xr, P.craw);
    spmv(P.Gtraw, yr.data(), aty.data());
    double atyinf = nrminf(aty), atynrm1 = nrm1(aty);
    for (int64_t j = 0; j < n; ++j) lam[j] = P.craw[j] - aty[j];
    double dobj_ = dot(P.hraw, yr);
    for (int64_t j = 0; j < P.nb; ++j)
      dobj_ += P.bl_fin[j] * std::max(0.0, lam[j]) + P.bu_fin[j] * std::min(0.0, lam[j]);
    double abs_gap = std::fabs(pobj_ - dobj_);
    double rel_gap = o.cpu_semantics ? abs_gap / (1.0 + std::fabs(pobj_) + std::fabs(dobj_))
                                     : abs_gap / (1.0 + std::max(std::fabs(pobj_), std::fabs(dobj_)));
    spmv(P.Graw, xr.data(), gx.data());
    double axinf = nrminf(gx), axnrm1 = nrm1(gx);
    for (int64_t i = 0; i < m; ++i) r[i] = gx[i] - P.hraw[i];
    pr = r;
    project_all(P.conb, pr.data(), nullptr, nullptr, nullptr);
    Vec presid(m);
    for (int64_t i = 0; i < m; ++i) presid[i] = pr[i] - r[i];
    pl = lam;
    project_all(P.slackb, pl.data(), nullptr, P.lam_l.data(), P.lam_u.data());
    double sinf = nrminf(pl), snrm1 = nrm1(pl);
    Vec dresid(n);
    for (int64_t j = 0; j < n; ++j) dresid[j] = pl[j] - lam[j];
    double l2p = nrm2(presid), linfp = nrminf(presid), l2d = nrm2(dresid), linfd = nrminf(dresid);
    C.pobj = pobj_;
    C.dobj = dobj_;
    C.abs_gap = abs_gap;
    C.rel_gap = rel_gap;
    C.l2_abs_p = l2p;
    C.linf_abs_p = linfp;
    C.l2_abs_d = l2d;
    C.linf_abs_d = linfd;
    if (o.cpu_semantics) {
      C.l2_rel_p = l2p / (1.0 + P.hNrm1);
      C.linf_rel_p = linfp / (1.0 + P.hNrmInf);
      C.l2_rel_d = l2d / (1.0 + P.cNrm1);
      C.linf_rel_d = linfd / (1.0 + P.cNrmInf);
    } else {
      C.l2_rel_p = l2p / (1.0 + std::max(snrm1, std::max(P.hNrm1, axnrm1)));
      C.linf_rel_p = linfp / (1.0 + std::max(sinf, std::max(P.hNrmInf, axinf)));
      C.l2_rel_d = l2d / (1.0 + std::max(P.cNrm1, atynrm1));
      C.linf_rel_d = linfd / (1.0 + std::max(P.cNrmInf, atyinf));
    }
  }

  // infeasibility_info_calculation_diagonal! (rpdhg_alg_gpu_gen_scaling.jl:185-248)
  void infeasibility_info(bool have_pobj, double pobj_in, const Vec& pray, const Vec& dray, Infea& I,
                          double pobj_seq, double dobj_seq) {
    double pobj_ = have_pobj ? pobj_in : dot(pray, P.craw);
    bool have_lp = false, have_ld = false;
    double lp = 0, ld = 0;
    if (pobj_ < 0.0) {
      Vec gx(m), pr(m);
      spmv(P.Graw, pray.data(), gx.data());
      for (int64_t i = 0; i < m; ++i) gx[i] -= P.hraw[i];
      pr = gx;
      project_all(P.conb, pr.data(), nullptr, nullptr, nullptr);
      for (int64_t i = 0; i < m; ++i) lp = std::max(lp, std::fabs(pr[i] - gx[i]));
      have_lp = true;
    }
    double dobj_ = dot(P.hraw, dray);
    Vec aty(n), lam(n);
    spmv(P.Gtraw, dray.data(), aty.data());
    for (int64_t j = 0; j < n; ++j) lam[j] = P.craw[j] - aty[j];
    for (int64_t j = 0; j < P.nb; ++j)
      dobj_ += P.bl_fin[j] * std::max(0.0, lam[j]) + P.bu_fin[j] * std::min(0.0, lam[j]);
    if (dobj_ > 0.0) {
      Vec pl = lam;
      project_all(P.slackb, pl.data(), nullptr, P.lam_l.data(), P.lam_u.data());
      for (int64_t j = 0; j < n; ++j) ld = std::max(ld, std::fabs(pl[j] - lam[j]));
      have_ld = true;
    }
    I.primal_ray_obj = pobj_;
    I.dual_ray_obj = dobj_;
    I.max_primal_ray_inf = have_lp ? lp : 1e10;
    I.max_dual_ray_inf = have_ld ? ld : 1e10;
    I.primal_ray_norm = nrminf(pray);
    I.dual_ray_norm = nrminf(dray);
    // the reference pushes with probability 1/4 (rand() < 0.25); here every fourth check
    if (check_count % 4 == 0) {
      I.ptrend.push_back(pobj_seq);
      I.dtrend.push_back(dobj_seq);
      if (I.ptrend.size() > 20) I.ptrend.erase(I.ptrend.begin());
      if (I.dtrend.size() > 20) I.dtrend.erase(I.dtrend.begin());
    }
  }

  static bool mono_inc(const std::vector<double>& b) {
    if (b.size() < 20) return false;
    for (size_t i = 1; i < 20; ++i) if (b[i] < b[i - 1]) return false;
    return true;
  }
  static bool mono_dec(const std::vector<double>& b) {
    if (b.size() < 20) return false;
    for (size_t i = 1; i < 20; ++i) if (b[i] > b[i - 1]) return false;
    return true;
  }

  // check_termination_criteria (src/pdcs_gpu/termination.jl:74-260)
  void check_termination() {
    for (int k = 0; k < 2; ++k) {
      Converge& C = ci[k];
      if (std::max(C.linf_rel_p, std::max(C.linf_rel_d, C.rel_gap)) < o.rel_tol) C.status = 0;
      if (std::max(C.linf_abs_p, std::max(C.linf_abs_d, C.abs_gap)) < o.abs_tol) C.status = 0;
      if (std::isnan(C.rel_gap)) C.status = 8;
      if (std::isinf(C.rel_gap)) C.status = 9;
      if (C.status == 0) {
        exit_code = 0;
        pobj = C.pobj;
        dobj = C.dobj;
        returned_seq = k;
        return;
      }
      if (C.status == 8 || C.status == 9) {
        exit_code = C.status;
        return;
      }
    }
    for (int k = 0; k < 2; ++k) {
      Infea& I = ii[k];
      // primal infeasibility (termination.jl:96-136)
      if (I.dual_ray_obj > 0.0) {
        if ((I.dual_ray_obj - I.primal_ray_obj) / (1 + std::fabs(I.dual_ray_obj) + std::fabs(I.primal_ray_obj)) > 0.99999 &&
            I.max_primal_ray_inf > 1e3 && mono_inc(I.dtrend) && I.max_dual_ray_inf > 1e4 &&
            I.dual_ray_obj > 1e14 && I.dual_ray_norm > 1e8)
          I.status = 2;
        double res = std::max(I.max_dual_ray_inf, 1.0) / I.dual_ray_obj;
        if (res <= o.eps_primal_infeasible_low_acc) {
          if (res <= o.eps_primal_infeasible_high_acc) I.status = 3;
          if (I.max_dual_ray_inf > 1e8) I.status = 2;
          if (mono_inc(I.dtrend)) I.status = 2;
        }
      }
      if (I.status == 2 && iter > 2000) { exit_code = 2; pobj = I.primal_ray_obj; dobj = I.dual_ray_obj; return; }
      if (I.status == 3 && iter > 500) { exit_code = 3; pobj = I.primal_ray_obj; dobj = I.dual_ray_obj; return; }
      // dual infeasibility (termination.jl:138-180)
      if (I.primal_ray_obj < 0.0) {
        if ((I.primal_ray_obj - I.dual_ray_obj) / (1 + std::fabs(I.primal_ray_obj) + std::fabs(I.dual_ray_obj)) > 0.99999 &&
            I.max_dual_ray_inf > 1e3 && mono_dec(I.ptrend) && I.max_primal_ray_inf > 1e4 &&
            -I.primal_ray_obj > 1e14 && I.primal_ray_norm > 1e8)
          I.status = 4;
        double res = std::max(I.max_primal_ray_inf, 1.0) / (-I.primal_ray_obj);
        if (res <= o.eps_dual_infeasible_low_acc) {
          if (res <= o.eps_dual_infeasible_high_acc) I.status = 5;
          if (I.max_primal_ray_inf > 1e8) I.status = 4;
          if (mono_dec(I.ptrend)) I.status = 4;
        }
      }
      if (I.status == 4 && iter > 2000) { exit_code = 4; pobj = I.primal_ray_obj; dobj = I.dual_ray_obj; return; }
      if (I.status == 5 && iter > 500) { exit_code = 5; pobj = I.primal_ray_obj; dobj = I.dual_ray_obj; return; }
    }
    if ((double)iter >= (double)o.max_outer_iter * (double)o.max_inner_iter) {
      exit_code = 1;
      pobj = ci[0].pobj;
      dobj = ci[0].dobj;
      return;
    }
    if (o.time_limit > 0 && now_s() - t_start > o.time_limit) {
      exit_code = 6;
      return;
    }
    exit_code = 7;
  }

  void recover(Vec& xr, Vec& xmr, Vec& yr, Vec& ymr) {
    for (int64_t j = 0; j < n; ++j) {
      xr[j] = x[j] / P.Dr[j];
      xmr[j] = xm[j] / P.Dr[j];
    }
    for (int64_t i = 0; i < m; ++i) {
      yr[i] = y[i] / P.Dl[i];
      ymr[i] = ym[i] / P.Dl[i];
    }
  }

  // exit_condition_check_diagonal! (rpdhg_alg_gpu_gen_scaling.jl:309-352)
  void exit_check() {
    Vec xr(n), xmr(n), yr(m), ymr(m);
    recover(xr, xmr, yr, ymr);
    converge_info(xr, yr, ci[0]);
    converge_info(xmr, ymr, ci[1]);
    infeasibility_info(true, ci[0].pobj, xr, yr, ii[0], ci[0].pobj, ci[0].dobj);
    Vec dx(n), dy(m);
    for (int64_t j = 0; j < n; ++j) dx[j] = xr[j] - xmr[j];
    for (int64_t i = 0; i < m; ++i) dy[i] = yr[i] - ymr[i];
    infeasibility_info(false, 0.0, dx, dy, ii[1], ci[0].pobj, ci[0].dobj);
    check_count++;
    check_termination();
  }

  // approximate_cal_diagonal! + binary_search_duality_gap_diagonal!
  // (rpdhg_alg_gpu_gen_scaling.jl:2-117).  The doubling loop's
  // `tRight = t, tLeft = t / 2, break` parses in Julia as
  // `tRight = ((t, tLeft) = (t / 2, break))`; the break runs while the right-hand
  // tuple is being built, so the loop exits with tLeft/tRight unchanged.
  double binary_search(double r, const Vec& px, const Vec& py, double ta, double si) {
    Vec& h1 = tn1;
    Vec& h2 = tm1;
    Vec& xs = tn2;
    Vec& ys = tm2;
    Vec dx(n), dy(m);
    spmv(P.Gt, py.data(), h1.data());
    for (int64_t j = 0; j < n; ++j) h1[j] -= P.c[j];
    spmv(P.G, px.data(), h2.data());
    for (int64_t i = 0; i < m; ++i) h2[i] = -h2[i] + P.h[i];
    auto approx = [&](double t) {
      for (int64_t j = 0; j < n; ++j) xs[j] = px[j] + (t * ta / 2) * h1[j];
      proj_x(xs.data());
      for (int64_t i = 0; i < m; ++i) ys[i] = py[i] + (t * si / 2) * h2[i];
      proj_y(ys.data());
      for (int64_t j = 0; j < n; ++j) dx[j] = xs[j] - px[j];
      for (int64_t i = 0; i < m; ++i) dy[i] = ys[i] - py[i];
      return mnorm(dx, dy, ta, si);
    };
    double t = bs_t0, tR = t, tL = 0.0;
    for (int k = 1; k <= 1000; ++k) {
      double val = approx(t);
      if (val > r && val < r + 1e-6) {
        tR = t;
        tL = std::max(t - 0.01, 0.0);
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
    }
    double tM = 0.5 * (tR + tL);
    int64_t count = 0;
    while (tR - tL > 1e-6) {
      tM = 0.5 * (tR + tL);
      if (approx(tM) < r) tL = tM; else tR = tM;
      if (++count > 1000000) break;
    }
    bs_t0 = tM;
    // calculate_diff uses the last evaluated projections
    return (dot(h1, dx) + dot(h2, dy)) / r;
  }

  // kkt_error_diagonal! (rpdhg_alg_gpu_gen_scaling.jl:119-122)
  double kkt_error(const Converge& C) const {
    return std::sqrt(omega * omega * C.l2_abs_p * C.l2_abs_p + C.l2_abs_d * C.l2_abs_d / (omega * omega) +
                     C.abs_gap * C.abs_gap);
  }

  // restart_threshold_calculation_diagonal! (rpdhg_alg_gpu_gen_scaling.jl:354-393)
  void restart_threshold(bool dgap) {
    if (dgap) {
      Vec dx(n), dy(m);
      for (int64_t j = 0; j < n; ++j) dx[j] = x0[j] - x0l[j];
      for (int64_t i = 0; i < m; ++i) dy[i] = y0[i] - y0l[i];
      double r = mnorm(dx, dy, tau, sigma);
      ndg_r = r;
      ndg_thr = binary_search(r, x0, y0, tau, sigma);
      if (ndg_thr < 0) dgap_flag = false;
    } else {
      Vec xr(n), xmr(n), yr(m), ymr(m);
      recover(xr, xmr, yr, ymr);
      converge_info(xr, yr, ci[0]);
      kkt_thr = kkt_error(ci[0]);
    }
  }

  void restart_to_current() {
    xm = x;
    ym = y;
  }

  // restart_condition_check_diagonal! (rpdhg_alg_gpu_gen_scaling.jl:395-506)
  bool restart_check(int64_t inner, bool dgap) {
    if (dgap) {
      Vec dx(n), dy(m);
      for (int64_t j = 0; j < n; ++j) dx[j] = x[j] - x0[j];
      for (int64_t i = 0; i < m; ++i) dy[i] = y[i] - y0[i];
      double rl = mnorm(dx, dy, tau, sigma);
      double rho = binary_search(rl, x, y, tau, sigma);
      double rho_m = binary_search(rl, xm, ym, tau, sigma);
      ndg[0] = rho;
      ndg[1] = rho_m;
      for (double beta : {beta_suff, beta_nec}) {
        if (rho < beta * ndg_thr || rho_m < beta * ndg_thr) {
          restart_used++;
          if (ndg[0] < ndg[1] && dgap_flag) {
            trig_ergodic++;
            restart_to_current();
          } else {
            trig_mean++;
          }
          return true;
        }
      }
    } else {
      Vec xr(n), xmr(n), yr(m), ymr(m);
      recover(xr, xmr, yr, ymr);
      converge_info(xr, yr, ci[0]);
      converge_info(xmr, ymr, ci[1]);
      double lag0 = kkt_err[0], lag1 = kkt_err[1];
      double e0 = kkt_error(ci[0]), e1 = kkt_error(ci[1]);
      kkt_err[0] = e0;
      kkt_err[1] = e1;
      bool c1 = e0 < beta_suff_kkt * kkt_thr || e1 < beta_suff_kkt * kkt_thr;
      bool c2 = (e0 < beta_nec_kkt * kkt_thr && e0 > lag0) || (e1 < beta_nec_kkt * kkt_thr && e1 > lag1);
      if (c1 || c2) {
        restart_used++;
        if (kkt_err[0] < kkt_err[1]) {
          trig_ergodic++;
          restart_to_current();
        } else {
          trig_mean++;
        }
        return true;
      }
    }
    if ((double)inner >= (double)iter * beta_art && iter > 100000) {
      restart_used++;
      return true;
    }
    return false;
  }

  void update_best() {
    if (ci[0].l2_rel_p < pres_best) {
      pres_best = ci[0].l2_rel_p;
      xbest = x;
    }
    if (ci[0].l2_rel_d < dres_best) {
      dres_best = ci[0].l2_rel_d;
      ybest = y;
    }
  }

  double init_omega() {
    double hn = nrm2(P.h), cn = nrm2(P.c);
    return (hn > 1e-10 && cn > 1e-10) ? cn / hn : 1.0;
  }

  double omega_update(const Vec& xd, const Vec& yd, double om) {
    double xn = nrm2(xd), yn = nrm2(yd);
    if ((om > 1e4 || om < 1e-4) && restart_used % 20 == 0 && restart_used != 0) return init_omega();
    if ((om > 3e4 || om < 1.0 / 3e4) && restart_used % 10 == 0 && restart_used != 0) return init_omega();
    if (xn > 1e-10 && yn > 1e-10) return std::exp(0.5 * std::log(yn / xn) + 0.5 * std::log(om));
    return om;
  }

  bool out_of_attempts() {
    if (o.attempt_limit > 0 && iter >= o.attempt_limit) {
      attempt_limit_hit = true;
      return true;
    }
    return false;
  }

  // pdhg_one_iter_diagonal_rescaling_adaptive_step_size!
  // (rpdhg_alg_gpu_gen_scaling.jl:656-766; CPU variant rpdhg_alg_cpu_gen_scaling.jl:685-766)
  // returns (eta, eta_prime, force_restart)
  void one_iter(double& eta, double& eta_p, bool& force) {
    force = false;
    eta = std::max(eta, 1e-6);
    xl = x;
    yl = y;
    double dec = o.cpu_semantics ? 1.0 : decay();
    Vec& aty = tn1;
    Vec& dxv = tn2;
    Vec& gdy = tn3;
    Vec& gxb = tm1;
    Vec& dyv = tm2;
    int64_t count = 0;
    while (true) {
      iter++;
      iter_stepsize++;
      spmv(P.Gt, yl.data(), aty.data());
      tau = eta / omega;
      double ps = tau * dec;
      for (int64_t j = 0; j < n; ++j) x[j] = xl[j] + ps * (aty[j] - P.c[j]);
      proj_x(x.data());
      for (int64_t j = 0; j < n; ++j) dxv[j] = 2.0 * x[j] - xl[j];
      spmv(P.G, dxv.data(), gxb.data());
      sigma = eta * omega;
      double ds = sigma * dec;
      for (int64_t i = 0; i < m; ++i) y[i] = yl[i] - ds * (gxb[i] - P.h[i]);
      proj_y(y.data());
      for (int64_t i = 0; i < m; ++i) dyv[i] = y[i] - yl[i];
      for (int64_t j = 0; j < n; ++j) dxv[j] = x[j] - xl[j];
      double num = omega * dot(dxv, dxv) + dot(dyv, dyv) / omega;
      spmv(P.Gt, dyv.data(), gdy.data());
      double den = 2.0 * std::fabs(dot(dxv, gdy));
      double eta_bar = num / (den + kPositiveZero);
      double k1 = (double)(iter_stepsize + 1);
      eta_p = std::min((1.0 - std::pow(k1, -0.3)) * eta_bar, (1.0 + std::pow(k1, -0.6)) * eta);
      if (iter % o.check_terminate_freq == 0) {
        exit_check();
        if (!o.cpu_semantics) {
          max_kkt = std::max(std::max(ci[0].l2_rel_p, ci[0].l2_rel_d), ci[0].rel_gap);
          double avg = (ci[0].l2_rel_p + ci[0].l2_rel_d + ci[0].rel_gap) / 3.0;
          proj_abs_tol = std::max(std::min(proj_abs_tol, std::min(avg * proj_base_tol, 1e-7)), 5e-16);
          proj_rel_tol = std::max(std::min(proj_rel_tol, std::min(avg * proj_base_tol, 1e-7)), 5e-16);
        }
        if (o.verbose)
          std::printf("[oracle] iter %lld rel_p %.3e rel_d %.3e gap %.3e pobj %.6e dobj %.6e restarts %lld"
                      " eta %.3e eta_bar %.3e omega %.3e |x| %.3e |y| %.3e\n",
                      (long long)iter, ci[0].linf_rel_p, ci[0].linf_rel_d, ci[0].rel_gap, ci[0].pobj, ci[0].dobj,
                      (long long)restart_used, eta, eta_bar, omega, nrm2(x), nrm2(y));
        if (exit_code != 7) return;
      }
      if (out_of_attempts()) return;
      bool accept = o.cpu_semantics ? (eta <= 0.99 * eta_bar) : (eta <= eta_bar);
      if (accept) return;
      eta = eta_p;
      if (++count > 1000000) {
        proj_abs_tol = std::max(proj_abs_tol * 0.1, 1e-22);
        proj_rel_tol = std::max(proj_rel_tol * 0.1, 1e-22);
        force = true;
        return;
      }
    }
  }

  // reflection_update (src/pdcs_gpu/cuda/utils.cu:37-56)
  void reflect(double extra, int64_t inner, double eta_cum, double eta) {
    double di = (double)inner;
    double tmp = (di + 1.0) / (di + 2.0);
    for (int64_t j = 0; j < n; ++j) {
      x[j] = tmp * ((1.0 + extra) * x[j] - extra * xl[j]) + (1.0 / (di + 2.0)) * x[j];
      xm[j] = (xm[j] * eta_cum + x[j] * eta) / (eta_cum + eta);
    }
    for (int64_t i = 0; i < m; ++i) {
      y[i] = tmp * ((1.0 + extra) * y[i] - extra * yl[i]) + (1.0 / (di + 2.0)) * y[i];
      ym[i] = (ym[i] * eta_cum + y[i] * eta) / (eta_cum + eta);
    }
  }

  double power_method(double* flag) {
    // power_method! (def_rpdhg_gen.jl:891-917), deterministic start vector
    Vec b(n), ab(m), atab(n);
    uint64_t st = 0x9E3779B97F4A7C15ull;
    for (int64_t j = 0; j < n; ++j) {
      st = st * 6364136223846793005ull + 1442695040888963407ull;
      b[j] = (double)(st >> 11) * (1.0 / 9007199254740992.0);
    }
    double nb_ = nrm2(b);
    for (auto& v : b) v /= nb_;
    double lam_old = 0.0, lam = 0.0;
    for (int it = 0; it < 1000; ++it) {
      spmv(P.G, b.data(), ab.data());
      spmv(P.Gt, ab.data(), atab.data());
      b = atab;
      nb_ = nrm2(b);
      for (auto& v : b) v /= nb_;
      spmv(P.G, b.data(), ab.data());
      spmv(P.Gt, ab.data(), atab.data());
      lam = dot(b, atab);
      if (std::fabs(lam - lam_old) < 1e-3) {
        *flag = 0;
        return std::sqrt(lam);
      }
      lam_old = lam;
    }
    *flag = 1;
    return std::sqrt(lam);
  }

  // resolving_pessimistic_step! (rpdhg_alg_gpu_gen_scaling.jl:511-638)
  void resolving() {
    iter_stepsize = 0;
    double flag;
    double gl = power_method(&flag);
    sigma = tau = (flag == 0 ? 0.9 : 0.8) / gl;
    omega = std::min(std::max(init_omega(), 0.8), 1.2);
    xm = xbest;
    ym = ybest;
    for (int64_t outer = 1; outer <= o.max_outer_iter; ++outer) {
      x0l = x0;
      y0l = y0;
      x0 = xm;
      y0 = ym;
      x = xm;
      y = ym;
      if (o.use_kkt_restart) restart_threshold(false);
      else restart_threshold(dgap_flag);
      int64_t inner = 0;
      Vec xd = x, yd = y;
      while (true) {
        inner++;
        iter++;
        // pdhg_one_iter_diagonal_rescaling! (:250-263)
        double ta = tau / omega, si = sigma * omega;
        xl = x;
        spmv(P.Gt, y.data(), tn1.data());
        for (int64_t j = 0; j < n; ++j) x[j] = xl[j] + ta * (tn1[j] - P.c[j]);
        proj_x(x.data());
        for (int64_t j = 0; j < n; ++j) xl[j] = 2.0 * x[j] - xl[j];
        spmv(P.G, xl.data(), tm1.data());
        for (int64_t i = 0; i < m; ++i) y[i] -= si * (tm1[i] - P.h[i]);
        proj_y(y.data());
        double di = (double)inner;
        for (int64_t j = 0; j < n; ++j) xm[j] = (xm[j] * di + x[j]) / (di + 1.0);
        for (int64_t i = 0; i < m; ++i) ym[i] = (ym[i] * di + y[i]) / (di + 1.0);
        // :570-596: the restart tests come first and break before the exit check
        if (iter % o.kkt_restart_freq == 0 && o.use_kkt_restart) {
          if (restart_check(inner, false) || outer == 1) break;
        }
        if (iter % o.duality_gap_restart_freq == 0 && o.use_duality_gap_restart) {
          if (restart_check(inner, dgap_flag) || outer == 1) break;
        }
        if (iter % o.check_terminate_freq == 0) {
          exit_check();
          if (exit_code != 7) return;
        }
        if (out_of_attempts()) return;
      }
      for (int64_t j = 0; j < n; ++j) xd[j] -= x[j];
      for (int64_t i = 0; i < m; ++i) yd[i] -= y[i];
      omega = std::min(std::max(omega_update(xd, yd, omega), 0.8), 1.2);
    }
    exit_code = 1;
  }

  // pdhg_main_iter_average_diagonal_rescaling_restarts_adaptive_weight_resolving_aggressive!
  // (rpdhg_alg_gpu_gen_scaling.jl:770-895)
  void main_loop() {
    x0 = x;
    y0 = y;
    x0l = x;
    y0l = y;
    omega = init_omega();
    double ginf = 0.0;
    for (double v : P.G.v) ginf = std::max(ginf, std::fabs(v));
    double eta_p = 1.0 / ginf;
    for (int64_t outer = 1; outer <= o.max_outer_iter; ++outer) {
      update_best();
      max_kkt = std::max(std::max(ci[0].l2_rel_p, ci[0].l2_rel_d), ci[0].rel_gap);
      min_kkt = std::min(std::min(std::min(ci[0].l2_rel_p, ci[0].l2_rel_d), ci[0].rel_gap), min_kkt);
      double extra = -0.1 * std::log10(max_kkt) + 0.2;
      x0l = x0;
      y0l = y0;
      x0 = xm;
      y0 = ym;
      x = xm;
      y = ym;
      if (o.use_kkt_restart) restart_threshold(false);
      else restart_threshold(dgap_flag);
      bool f1 = outer > 10 && max_kkt > 1e5;
      double pd = ci[0].l2_rel_p / ci[0].l2_rel_d;
      bool f2 = outer > 80 && (pd > 1e10 || pd < 1e-10);
      bool f3 = outer > 10 && tau < 1e-6 && sigma < 1e-6;
      bool f4 = iter > 1000000 && ci[0].rel_gap > 0.98 && ci[0].l2_rel_p > 1.0 && ci[0].l2_rel_d > 1.0;
      if (f1 || f2 || f3 || f4 || o.force_resolving) {
        resolving();
        return;
      }
      int64_t inner = 0;
      Vec xd = x, yd = y;
      double eta_cum = 0.0;
      while (true) {
        inner++;
        double eta = eta_p;  // the step is called with eta = eta_prime (:845-850)
        bool force;
        one_iter(eta, eta_p, force);
        if (exit_code != 7 || attempt_limit_hit) return;
        eta = std::max(eta, 1e-30);
        reflect(extra, inner, eta_cum, eta);
        eta_cum += eta;
        if (((double)inner >= (double)iter * beta_art && iter > 10000) || (force && inner > 100)) {
          restart_used++;
          break;
        }
        if (iter % o.kkt_restart_freq == 0 && o.use_kkt_restart) {
          if (restart_check(inner, false)) break;
          if (outer == 1) break;
        }
        if (iter % o.duality_gap_restart_freq == 0 && o.use_duality_gap_restart) {
          if (restart_check(inner, dgap_flag)) break;
          if (outer == 1) break;
        }
      }
      for (int64_t j = 0; j < n; ++j) xd[j] -= x[j];
      for (int64_t i = 0; i < m; ++i) yd[i] -= y[i];
      omega = omega_update(xd, yd, omega);
    }
    exit_code = 1;
  }
};

}  // namespace

extern "C" {

void oracle_default_options(oracle_options* o) {
  std::memset(o, 0, sizeof(*o));
  o->max_outer_iter = 10000;
  o->max_inner_iter = 500000;
  o->abs_tol = 1e-6;
  o->rel_tol = 1e-6;
  o->eps_primal_infeasible_low_acc = 1e-12;
  o->eps_dual_infeasible_low_acc = 1e-12;
  o->eps_primal_infeasible_high_acc = 1e-16;
  o->eps_dual_infeasible_high_acc = 1e-16;
  o->check_terminate_freq = 2000;
  o->kkt_restart_freq = 2000;
  o->duality_gap_restart_freq = 2000;
  o->use_kkt_restart = 0;
  o->use_duality_gap_restart = 1;
  o->rescaling = 3;
  o->cpu_semantics = 0;
  o->threads = 0;
  o->verbose = 0;
  o->time_limit = 0;
  o->attempt_limit = 0;
  o->warm_x = nullptr;
  o->warm_y = nullptr;
  o->force_resolving = 0;
}

int oracle_project_block(int kind, double* v, int64_t len, const double* S, const double* lo,
                         const double* hi) {
  return project_block(kind, v, len, S, lo, hi);
}

void oracle_proj_exp_scaled(double* v, const double* D) { proj_exp_scaled_impl(v, D); }

int oracle_precondition(const oracle_problem* p, int rescaling, double* Dr, double* Dl, double* scaled_val) {
  Problem P;
  int rc = build_problem(p, rescaling, P);
  if (rc) return rc;
  std::memcpy(Dr, P.Dr.data(), sizeof(double) * P.n);
  std::memcpy(Dl, P.Dl.data(), sizeof(double) * P.m);
  std::memcpy(scaled_val, P.G.v.data(), sizeof(double) * P.G.v.size());
  return 0;
}

// Shared FP64 evaluator of a final point (x, y) in the original scale.
// out[0] primal residual, README form: ||r - P(r)||_inf / (1 + max(||h||, ||Gx||, ||P(r)||)), r = Gx - h
// out[1] dual residual: ||lam - P(lam)||_inf / (1 + max(||c||, ||G'y||)), lam = c - G'y
// out[2] relative gap |c'x - dobj| / (1 + max(|c'x|, |dobj|)), dobj = h'y + l'lam+ + u'lam-
// out[3] primal residual with the GPU code's denominator (||P(lam)|| instead of ||P(r)||)
// out[4] c'x, out[5] dobj, out[6] ||r - P(r)||_inf, out[7] ||lam - P(lam)||_inf
// (README.md:70-90; rpdhg_alg_gpu_gen_scaling.jl:126-183)
int oracle_evaluate(const oracle_problem* p, const double* x, const double* y, double* out) {
  Problem P;
  int rc = build_problem(p, 0, P);
  if (rc) return rc;
  int64_t n = p->n, m = p->m;
  Vec xv(x, x + n), yv(y, y + m), gx(m), aty(n), r(m), pr(m), lam(n), pl(n);
  spmv(P.Graw, xv.data(), gx.data());
  spmv(P.Gtraw, yv.data(), aty.data());
  for (int64_t i = 0; i < m; ++i) r[i] = gx[i] - P.hraw[i];
  pr = r;
  project_all(P.conb, pr.data(), nullptr, nullptr, nullptr);
  for (int64_t j = 0; j < n; ++j) lam[j] = P.craw[j] - aty[j];
  pl = lam;
  project_all(P.slackb, pl.data(), nullptr, P.lam_l.data(), P.lam_u.data());
  double rinf = 0, linf = 0;
  for (int64_t i = 0; i < m; ++i) rinf = std::max(rinf, std::fabs(pr[i] - r[i]));
  for (int64_t j = 0; j < n; ++j) linf = std::max(linf, std::fabs(pl[j] - lam[j]));
  double pobj = dot(xv, P.craw), dobj = dot(yv, P.hraw);
  for (int64_t j = 0; j < P.nb; ++j)
    dobj += P.bl_fin[j] * std::max(0.0, lam[j]) + P.bu_fin[j] * std::min(0.0, lam[j]);
  double hinf = nrminf(P.hraw), gxinf = nrminf(gx), prinf = nrminf(pr), cinf = nrminf(P.craw);
  double atyinf = nrminf(aty), plinf = nrminf(pl);
  out[0] = rinf / (1.0 + std::max(hinf, std::max(gxinf, prinf)));
  out[1] = linf / (1.0 + std::max(cinf, atyinf));
  out[2] = std::fabs(pobj - dobj) / (1.0 + std::max(std::fabs(pobj), std::fabs(dobj)));
  out[3] = rinf / (1.0 + std::max(plinf, std::max(hinf, gxinf)));
  out[4] = pobj;
  out[5] = dobj;
  out[6] = rinf;
  out[7] = linf;
  return 0;
}

int oracle_solve(const oracle_problem* p, const oracle_options* opt, oracle_result* res) {
#ifdef _OPENMP
  if (opt->threads > 0) omp_set_num_threads(opt->threads);
#endif
  double t0 = now_s();
  Solver S;
  S.o = *opt;
  int rc = build_problem(p, opt->rescaling, S.P);
  if (rc) return rc;
  S.n = p->n;
  S.m = p->m;
  S.x.assign(S.n, 0.0);
  S.y.assign(S.m, 0.0);
  if (opt->warm_x)
    for (int64_t j = 0; j < S.n; ++j) S.x[j] = opt->warm_x[j] * S.P.Dr[j];
  if (opt->warm_y)
    for (int64_t i = 0; i < S.m; ++i) S.y[i] = opt->warm_y[i] * S.P.Dl[i];
  S.xl = S.x;
  S.xm = S.x;
  S.yl = S.y;
  S.ym = S.y;
  S.xbest = S.x;
  S.ybest = S.y;
  for (Vec* v : {&S.tn1, &S.tn2, &S.tn3}) v->assign(S.n, 0.0);
  for (Vec* v : {&S.tm1, &S.tm2, &S.tm3}) v->assign(S.m, 0.0);
  // initial convergence information (rpdhg_alg_gpu_gen.jl:1865-1881)
  {
    Vec xr(S.n), xmr(S.n), yr(S.m), ymr(S.m);
    S.recover(xr, xmr, yr, ymr);
    S.converge_info(xr, yr, S.ci[0]);
  }
  S.t_start = now_s();
  res->setup_seconds = S.t_start - t0;
  S.main_loop();
  res->solve_seconds = now_s() - S.t_start;
  if (S.attempt_limit_hit) S.exit_code = 10;
  Vec xr(S.n), xmr(S.n), yr(S.m), ymr(S.m);
  S.recover(xr, xmr, yr, ymr);
  const Vec& xo = (S.exit_code == 0 && S.returned_seq == 1) ? xmr : xr;
  const Vec& yo = (S.exit_code == 0 && S.returned_seq == 1) ? ymr : yr;
  if (res->x) std::memcpy(res->x, xo.data(), sizeof(double) * S.n);
  if (res->y) std::memcpy(res->y, yo.data(), sizeof(double) * S.m);
  const Converge& C = S.ci[S.exit_code == 0 ? S.returned_seq : 0];
  res->primal_objective = C.pobj;
  res->dual_objective = C.dobj;
  res->l_inf_rel_primal_res = C.linf_rel_p;
  res->l_inf_rel_dual_res = C.linf_rel_d;
  res->rel_gap = C.rel_gap;
  res->l_2_rel_primal_res = C.l2_rel_p;
  res->l_2_rel_dual_res = C.l2_rel_d;
  res->iter = S.iter;
  res->restart_used = S.restart_used;
  res->exit_code = S.exit_code;
  res->returned_sequence = S.returned_seq;
  return 0;
}

}  // extern "C"
