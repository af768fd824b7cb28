// pdcs_adjoint.cuh -- kernels of the solution-map adjoint (implicit
// differentiation of the PDHG fixed point).
//
// The solution z* = (x*, y*) of the unscaled problem is a fixed point of the
// PDHG map T(z) (x+ = P_X(x + T (G'y - c)), y+ = P_K*(y - S (G(2x+ - x) - h)))
// for positive diagonal steps T, S that are constant on every cone block (the
// optimality conditions are invariant to a positive scale per block).  The
// steps are Pock-Chambolle's, 0.9 / (column or row absolute sum), at their
// minimum over each block.  With M = dT/dz at z*, a loss gradient g = dL/dz*
// pulls back through u = (I - M)^{-T} g; applying M' needs one product with
// G and one with G' and the Jacobians D of the projections at the points
// a = x + T (G'y - c) (primal cones X) and b = y - S (Gx - h) (dual cones K*):
//   w = D_K u_y,  t = G' (S w),  q = u_x - 2 t,  r = D_X q,
//   M' u = (r + t,  w + G (T r)),
// and the parameter gradients follow from the same vectors:
//   dL/dc = -T r, dL/dh = S w, dL/dG_ij = T_j y_i r_j - S_i w_i x_j,
//   dL/dl = q [a < l], dL/du = q [a > u].
#pragma once
#include "pdcs_batch_kernels.cuh"

namespace pdcs {

// ---- projection Jacobians (unscaled cones) ----

// D v for the exponential cone at point a (cl{(r,s,t): s > 0, s e^{r/s} <= t}).
// Regions: a in K (D = I); polar (D = 0); r <= 0, s <= 0 (P = (r, 0, max(t, 0)));
// otherwise P(a) = p on the surface phi(p) = s e^{r/s} - t = 0 and, from the
// projection's optimality conditions (I + mu Hphi) dp + grad phi dmu = da,
// grad phi' dp = 0:  D = B^-1 - (B^-1 g)(B^-1 g)' / (g' B^-1 g), B = I + mu Hphi.
__device__ inline void exp_jac_apply(const double a[3], const double v[3], double out[3]) {
  double p0 = a[0], p1 = a[1], p2 = a[2];
  proj_exp_scaled_dev(p0, p1, p2, 1.0, 1.0, 1.0, nullptr);
  const double scale = 1.0 + sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  const double d0 = p0 - a[0], d1 = p1 - a[1], d2 = p2 - a[2];
  if (sqrt(d0 * d0 + d1 * d1 + d2 * d2) <= 1e-13 * scale) {
    out[0] = v[0]; out[1] = v[1]; out[2] = v[2];
    return;
  }
  if (sqrt(p0 * p0 + p1 * p1 + p2 * p2) <= 1e-13 * scale) {
    out[0] = out[1] = out[2] = 0.0;
    return;
  }
  if (p1 <= 1e-13 * scale) {
    out[0] = v[0];
    out[1] = 0.0;
    out[2] = a[2] > 0.0 ? v[2] : 0.0;
    return;
  }
  const double rho = p0 / p1, e = exp(rho);
  const double g[3] = {e, e * (1.0 - rho), -1.0};
  const double gg = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
  const double mu = -(d0 * g[0] + d1 * g[1] + d2 * g[2]) / gg;  // a - p = mu grad phi
  const double hs = mu * e / p1;
  // B = I + hs [[1, -rho, 0], [-rho, rho^2, 0], [0, 0, 0]]: invert the leading 2x2 block
  const double b00 = 1.0 + hs, b01 = -hs * rho, b11 = 1.0 + hs * rho * rho;
  const double det = b00 * b11 - b01 * b01;
  const double i00 = b11 / det, i01 = -b01 / det, i11 = b00 / det;
  auto binv = [&](const double x[3], double y[3]) {
    y[0] = i00 * x[0] + i01 * x[1];
    y[1] = i01 * x[0] + i11 * x[1];
    y[2] = x[2];
  };
  double bg[3], bv[3];
  binv(g, bg);
  binv(v, bv);
  const double gbg = g[0] * bg[0] + g[1] * bg[1] + g[2] * bg[2];
  const double gbv = g[0] * bv[0] + g[1] * bv[1] + g[2] * bv[2];  // = bg' v (B symmetric)
  for (int i = 0; i < 3; ++i) out[i] = bv[i] - bg[i] * gbv / gbg;
}

// out = D v over a cone table (kinds, bounds; no scaling), for the elements of
// the masked instances (mask NULL: all).  A warp per SOC / RSOC block, a thread
// per exponential cone; grid: T.ctaA + nwc_ctas + T.ctaC.
__global__ void __launch_bounds__(kThreads) jac_kernel(ConeTable T, int nwc_ctas, const double* __restrict__ a,
                                                      const double* __restrict__ v, double* __restrict__ out,
                                                      const int32_t* __restrict__ inst,
                                                      const uint8_t* __restrict__ mask) {
  const int b = blockIdx.x;
  auto live = [&](int64_t j) { return !mask || mask[inst[j]]; };
  if (b < T.ctaA) {
    const int64_t stride = (int64_t)T.ctaA * kThreads;
    for (int s = 0; s < T.nseg; ++s) {
      const int64_t j0 = T.seg_start[s], j1 = j0 + T.seg_len[s];
      const int32_t kind = T.seg_kind[s];
      for (int64_t j = j0 + (int64_t)b * kThreads + threadIdx.x; j < j1; j += stride) {
        if (!live(j)) continue;
        const double aj = a[j];
        bool pass;
        switch (kind) {
          case PK_ZERO: pass = false; break;
          case PK_NONNEG: pass = aj > 0.0; break;
          case PK_BOX: pass = aj > T.lo[j] && aj < T.hi[j]; break;
          default: pass = true; break;
        }
        out[j] = pass ? v[j] : 0.0;
      }
    }
  } else if (b < T.ctaA + nwc_ctas) {
    const int lane = threadIdx.x & 31;
    const double r2 = 0.7071067811865476;
    for (int64_t k = (int64_t)(b - T.ctaA) * kWarps + (threadIdx.x >> 5); k < T.nwc; k += (int64_t)nwc_ctas * kWarps) {
      const int64_t st = T.wc_start[k];
      if (!live(st)) continue;  // warp-uniform
      const int d = T.wc_len[k];
      const bool rsoc = T.wc_kind[k] == PK_RSOC;
      // RSOC: rotate (a, v) to the SOC form in the first two coordinates
      auto rot = [&](const double* src, int64_t i) {
        if (!rsoc || i >= 2) return src[st + i];
        return i == 0 ? (src[st] + src[st + 1]) * r2 : (src[st] - src[st + 1]) * r2;
      };
      double nx2 = 0.0;
      for (int i = 1 + lane; i < d; i += 32) {
        const double ai = rot(a, i);
        nx2 += ai * ai;
      }
      const double nx = sqrt(warp_sum_bcast(nx2));
      const double t = rot(a, 0);
      double out0 = 0.0;
      if (nx <= t) {  // interior: D = I
        for (int i = lane; i < d; i += 32) out[st + i] = v[st + i];
        continue;
      }
      if (nx <= -t) {  // polar: D = 0
        for (int i = lane; i < d; i += 32) out[st + i] = 0.0;
        continue;
      }
      // D = 1/2 [[1, xh'], [xh, (1 + t/|x|) I - (t/|x|) xh xh']]
      double xv = 0.0;
      for (int i = 1 + lane; i < d; i += 32) xv += rot(a, i) * rot(v, i);
      const double xhv = warp_sum_bcast(xv) / nx;
      const double v0 = rot(v, 0), ratio = t / nx;
      out0 = 0.5 * (v0 + xhv);
      double o1 = 0.0;  // rotated output of coordinate 1 (lane 0; needed to rotate back)
      for (int i = 1 + lane; i < d; i += 32) {
        const double xh = rot(a, i) / nx;
        const double o = 0.5 * (v0 * xh + (1.0 + ratio) * rot(v, i) - ratio * xh * xhv);
        if (rsoc && i == 1) o1 = o;
        else out[st + i] = o;
      }
      if (rsoc) {  // lane 0 holds rotated coordinates 0 and 1: rotate back
        if (lane == 0) {
          out[st] = (out0 + o1) * r2;
          out[st + 1] = (out0 - o1) * r2;
        }
      } else if (lane == 0) {
        out[st] = out0;
      }
    }
  } else {
    const int64_t total = T.exp_count + T.dexp_count;
    const int64_t tstride = (int64_t)T.ctaC * kThreads;
    for (int64_t k = (int64_t)(b - T.ctaA - nwc_ctas) * kThreads + threadIdx.x; k < total; k += tstride) {
      const bool first = k < T.exp_count;
      const int64_t j = first ? T.exp_base + 3 * k : T.dexp_base + 3 * (k - T.exp_count);
      if (!live(j)) continue;
      const int32_t kind = first ? T.exp_kind : T.dexp_kind;
      double aa[3] = {a[j], a[j + 1], a[j + 2]}, vv[3] = {v[j], v[j + 1], v[j + 2]}, oo[3];
      if (kind == PK_EXP) {
        exp_jac_apply(aa, vv, oo);
      } else {  // dual cone, Moreau: P_{K*}(a) = a + P_K(-a) => D* = I - D_K(-a)
        const double na[3] = {-aa[0], -aa[1], -aa[2]};
        exp_jac_apply(na, vv, oo);
        for (int i = 0; i < 3; ++i) oo[i] = vv[i] - oo[i];
      }
      out[j] = oo[0];
      out[j + 1] = oo[1];
      out[j + 2] = oo[2];
    }
  }
}

// ---- batched Krylov helpers on z = [x (n) | y (m)] (instance runs: rx, ry + n) ----

__device__ __forceinline__ int32_t inst_of_z(int64_t i, int64_t n, const int32_t* ix, const int32_t* iy) {
  return i < n ? ix[i] : iy[i - n];
}

// out[k * ld + p] = <V_p, w> over instance k's elements, p = p0 .. p0 + np - 1 (np <= 8);
// Per-instance dot products <V_{p0+p}, w> (p < np <= 8), split over S CTAs per
// instance: CTA (k, s) sums the instance's elements s, s + S, ... (in blocks of
// kThreads) into part[(k * S + s) * 8 + p]; adj_dots_reduce_kernel adds the S
// partials in order, so the result does not depend on scheduling.
__global__ void __launch_bounds__(kThreads) adj_dots_kernel(int64_t K, int S, const uint8_t* __restrict__ mask,
                                                           RunTable rx, RunTable ry, int64_t n,
                                                           const double* __restrict__ V, int64_t ldV, int p0, int np,
                                                           const double* __restrict__ w, double* __restrict__ part) {
  __shared__ double sh[8][kWarps];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int64_t ks = blockIdx.x; ks < K * S; ks += gridDim.x) {
    const int64_t k = ks / S;
    const int s = (int)(ks % S);
    if (mask && !mask[k]) continue;  // CTA-uniform
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int side = 0; side < 2; ++side) {
      const RunTable& rt = side ? ry : rx;
      const int64_t off = side ? n : 0;
      for (int q = 0; q < kMaxRuns; ++q) {
        const int64_t s0 = off + rt.start[k * kMaxRuns + q], L = rt.len[k * kMaxRuns + q];
        for (int64_t i = s0 + (int64_t)s * kThreads + threadIdx.x; i < s0 + L; i += (int64_t)S * kThreads) {
          const double wi = w[i];
#pragma unroll
          for (int p = 0; p < 8; ++p)
            if (p < np) acc[p] = fma(V[(int64_t)(p0 + p) * ldV + i], wi, acc[p]);
        }
      }
    }
#pragma unroll
    for (int p = 0; p < 8; ++p) {
      double v = acc[p];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
      if (lane == 0) sh[p][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < np) {
      double v = 0.0;
      for (int q = 0; q < kWarps; ++q) v += sh[threadIdx.x][q];
      part[ks * 8 + threadIdx.x] = v;
    }
    __syncthreads();
  }
}

__global__ void adj_dots_reduce_kernel(int64_t K, int S, const uint8_t* __restrict__ mask, int p0, int np,
                                       const double* __restrict__ part, double* __restrict__ out, int ld) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < K * np; t += stride) {
    const int64_t k = t / np;
    const int p = (int)(t % np);
    if (mask && !mask[k]) continue;
    double v = 0.0;
    for (int s = 0; s < S; ++s) v += part[(k * S + s) * 8 + p];
    out[k * ld + p0 + p] = v;
  }
}

// w[i] += sgn * sum_{p < np} coef[k * ld + p] V_p[i] on the masked instances' elements
__global__ void adj_combine_kernel(int64_t N, int64_t n, const int32_t* __restrict__ ix, const int32_t* __restrict__ iy,
                                   const uint8_t* __restrict__ mask, const double* __restrict__ V, int64_t ldV, int np,
                                   const double* __restrict__ coef, int ld, double sgn, double* __restrict__ w) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
    const int32_t k = inst_of_z(i, n, ix, iy);
    if (mask && !mask[k]) continue;
    double s = 0.0;
    for (int p = 0; p < np; ++p) s = fma(coef[(int64_t)k * ld + p], V[(int64_t)p * ldV + i], s);
    w[i] += sgn * s;
  }
}

// out[i] = a[k] * u[i] (per-instance scale) on the masked instances' elements
__global__ void adj_scale_kernel(int64_t N, int64_t n, const int32_t* __restrict__ ix, const int32_t* __restrict__ iy,
                                 const uint8_t* __restrict__ mask, const double* __restrict__ a,
                                 const double* __restrict__ u, double* __restrict__ out) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
    const int32_t k = inst_of_z(i, n, ix, iy);
    if (mask && !mask[k]) continue;
    out[i] = a[k] * u[i];
  }
}

// out = d * u (elementwise)
__global__ void adj_mul_kernel(int64_t len, const double* __restrict__ d, const double* __restrict__ u,
                               double* __restrict__ out) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += stride) out[i] = d[i] * u[i];
}

// q = ux - 2 t  (x side, masked)
__global__ void adj_q_kernel(int64_t n, const int32_t* __restrict__ ix, const uint8_t* __restrict__ mask,
                             const double* __restrict__ ux, const double* __restrict__ t, double* __restrict__ q) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
    if (mask && !mask[ix[j]]) continue;
    q[j] = ux[j] - 2.0 * t[j];
  }
}

// out = u - M'u: out_x = ux - (r + t), out_y = uy - (w + s)   (s = G (T r))
__global__ void adj_finish_kernel(int64_t n, int64_t m, const int32_t* __restrict__ ix, const int32_t* __restrict__ iy,
                                  const uint8_t* __restrict__ mask, const double* __restrict__ u,
                                  const double* __restrict__ r, const double* __restrict__ t,
                                  const double* __restrict__ w, const double* __restrict__ s,
                                  double* __restrict__ out) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n + m; i += stride) {
    if (i < n) {
      if (mask && !mask[ix[i]]) continue;
      out[i] = u[i] - (r[i] + t[i]);
    } else {
      const int64_t j = i - n;
      if (mask && !mask[iy[j]]) continue;
      out[i] = u[i] - (w[j] + s[j]);
    }
  }
}

// projection points: out = base + sgn * d * (prod - off)
__global__ void adj_point_kernel(int64_t len, const double* __restrict__ d, const double* __restrict__ base,
                                 const double* __restrict__ prod, const double* __restrict__ off, double sgn,
                                 double* __restrict__ out) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += stride)
    out[i] = base[i] + sgn * d[i] * (prod[i] - off[i]);
}

// steps 0.9 / absolute sum (1 where the sum is 0), then their minimum over every
// SOC / RSOC / exp block of the table (elementwise segments keep their own)
__global__ void adj_steps_kernel(int64_t len, double* __restrict__ d) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += stride)
    d[i] = d[i] > 0.0 ? 0.9 / d[i] : 1.0;
}

__global__ void adj_block_min_kernel(ConeTable T, double* __restrict__ d) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t k = gw; k < T.nwc; k += nw) {
    const int64_t st = T.wc_start[k];
    const int len = T.wc_len[k];
    double v = 1e308;
    for (int i = lane; i < len; i += 32) v = fmin(v, d[st + i]);
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(kFull, v, o));
    for (int i = lane; i < len; i += 32) d[st + i] = v;
  }
  const int64_t total = T.exp_count + T.dexp_count;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = k < T.exp_count ? T.exp_base + 3 * k : T.dexp_base + 3 * (k - T.exp_count);
    const double v = fmin(d[j], fmin(d[j + 1], d[j + 2]));
    d[j] = d[j + 1] = d[j + 2] = v;
  }
}

// One GMRES step's Hessenberg column, a thread per instance still extending its
// Krylov basis (mask): H(i, j) = h1_i + h2_i for i <= j (the two classical
// Gram-Schmidt passes), H(j+1, j) = |w|; the instance's earlier Givens
// rotations applied to the column, a new rotation that zeroes H(j+1, j), the
// rotated right-hand side gamma and the residual estimate |gamma_{j+1}| / beta0.
// An instance whose estimate reaches tol (or whose basis breaks down: the
// current iterate solves the system) leaves the mask, so the next step's
// kernels skip it.  Layouts: H per instance (mr + 1) x mr row-major, cs / sn
// per instance mr, gamma per instance mr + 1, the step's dot products at
// k * ld + i.
__global__ void adj_givens_kernel(int64_t K, int j, int mr, int ld, uint8_t* __restrict__ mask,
                                  const double* __restrict__ h1, const double* __restrict__ h2,
                                  const double* __restrict__ hn, double* __restrict__ H, double* __restrict__ cs,
                                  double* __restrict__ sn, double* __restrict__ gam,
                                  const double* __restrict__ beta0, double tol, int32_t* __restrict__ jk,
                                  int64_t* __restrict__ iters, double* __restrict__ res) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < K; k += stride) {
    if (!mask[k]) continue;
    double* Hk = H + (size_t)k * (mr + 1) * mr;
    double* ck = cs + (size_t)k * mr;
    double* sk = sn + (size_t)k * mr;
    double* gk = gam + (size_t)k * (mr + 1);
    const double hnk = sqrt(hn[k * ld]);
    for (int i = 0; i <= j; ++i) Hk[i * mr + j] = h1[k * ld + i] + h2[k * ld + i];
    Hk[(j + 1) * mr + j] = hnk;
    for (int i = 0; i < j; ++i) {
      const double a0 = Hk[i * mr + j], a1 = Hk[(i + 1) * mr + j];
      Hk[i * mr + j] = ck[i] * a0 + sk[i] * a1;
      Hk[(i + 1) * mr + j] = -sk[i] * a0 + ck[i] * a1;
    }
    const double a0 = Hk[j * mr + j], a1 = Hk[(j + 1) * mr + j];
    const double rr = hypot(a0, a1);
    const double c = rr > 0.0 ? a0 / rr : 1.0, s = rr > 0.0 ? a1 / rr : 0.0;
    ck[j] = c;
    sk[j] = s;
    Hk[j * mr + j] = rr;
    Hk[(j + 1) * mr + j] = 0.0;
    const double gj = gk[j];
    gk[j + 1] = -s * gj;
    gk[j] = c * gj;
    jk[k] = j + 1;
    iters[k]++;
    res[k] = fabs(gk[j + 1]) / beta0[k];
    if (res[k] <= tol || hnk <= 1e-300) mask[k] = 0;
  }
}

// End of a GMRES cycle, a thread per instance of the cycle (run): the
// coefficients y = H^{-1} gamma of its jk Krylov vectors by back substitution
// (coef[k * ld + q], zero for q >= jk).
__global__ void adj_backsub_kernel(int64_t K, int mr, int ld, const uint8_t* __restrict__ run,
                                   const int32_t* __restrict__ jk, const double* __restrict__ H,
                                   const double* __restrict__ gam, double* __restrict__ coef) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < K; k += stride) {
    double* y = coef + k * ld;
    const int J = run[k] ? jk[k] : 0;
    for (int q = J; q < ld; ++q) y[q] = 0.0;
    const double* Hk = H + (size_t)k * (mr + 1) * mr;
    const double* gk = gam + (size_t)k * (mr + 1);
    for (int i = J - 1; i >= 0; --i) {
      double v = gk[i];
      for (int q = i + 1; q < J; ++q) v -= Hk[i * mr + q] * y[q];
      y[i] = v / Hk[i * mr + i];
    }
  }
}

// w[i] *= 1 / sqrt(nrm2[k * ld]) on the masked instances' elements (Arnoldi normalisation)
__global__ void adj_normalize_kernel(int64_t N, int64_t n, const int32_t* __restrict__ ix,
                                     const int32_t* __restrict__ iy, const uint8_t* __restrict__ mask,
                                     const double* __restrict__ nrm2, int ld, double* __restrict__ w) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
    const int32_t k = inst_of_z(i, n, ix, iy);
    if (mask && !mask[k]) continue;
    const double s = nrm2[(int64_t)k * ld];
    if (s > 0.0) w[i] *= 1.0 / sqrt(s);
  }
}

// dG[e] = T_j y_i r_j - S_i w_i x_j over the stored entries (warp per row)
__global__ void adj_dG_kernel(int64_t m, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                              const double* __restrict__ Tx, const double* __restrict__ Sy,
                              const double* __restrict__ y, const double* __restrict__ w,
                              const double* __restrict__ x, const double* __restrict__ r, double* __restrict__ dG) {
  const int lane = threadIdx.x & 31;
  const int64_t wstride = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < m; i += wstride) {
    const double yi = y[i], sw = Sy[i] * w[i];
    for (int32_t e = rp[i] + lane; e < rp[i + 1]; e += 32) {
      const int32_t j = ci[e];
      dG[e] = Tx[j] * yi * r[j] - sw * x[j];
    }
  }
}

// dc = -T r;  dl = q [a < l], du = q [a > u] on the box part (first nb elements)
__global__ void adj_dc_kernel(int64_t n, int64_t nb, const double* __restrict__ Tx, const double* __restrict__ r,
                              const double* __restrict__ q, const double* __restrict__ a,
                              const double* __restrict__ lo, const double* __restrict__ hi,
                              double* __restrict__ dc, double* __restrict__ dl, double* __restrict__ du) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
    dc[j] = -Tx[j] * r[j];
    if (j < nb) {
      dl[j] = a[j] < lo[j] ? q[j] : 0.0;
      du[j] = a[j] > hi[j] ? q[j] : 0.0;
    }
  }
}

}  // namespace pdcs
