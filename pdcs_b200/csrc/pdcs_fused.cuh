// pdcs_fused.cuh -- fused tile kernels of the batched iteration graph.
//
// One PDHG attempt of the batch is two matrix passes.  A tile is a range of
// one instance's rows (its own row order across the type runs) cut only at
// cone boundaries, so every cone of the tile's rows lies inside the tile.  Its
// CTA
//   1. stages the instance's column segment in shared memory (y_lag for G',
//      the (x, x_lag) pairs for G),
//   2. runs the tile's rows in SELL-32 layout: the rows sorted by length and
//      cut into slices of 32, each slice stored column-major and padded to
//      its longest row, so a warp streams a slice with one coalesced load per
//      column (lane = row) and every gather is a shared-memory read; the
//      products land in shared memory,
//   3. finishes the primal (G') or dual (G) step of those rows: the update,
//      the projection onto the instance's cones (elementwise rows a thread
//      each, SOC / RSOC blocks of at most 32 elements in lane groups,
//      exponential cones a thread each) and the tile's partial sums of the
//      control step's reductions, written once per tile.
// The products never reach HBM and no per-element contribution is stored:
// the control kernel sums an instance's tile partials in tile order.
// (rpdhg_alg_gpu_gen_scaling.jl:680-714: the two SpMVs, primal_update,
// dual_update, the projections and the norms of one adaptive-step attempt.)
#pragma once
#include "pdcs_tiles.cuh"

namespace pdcs {

constexpr int kFusedThreads = 256;
constexpr int kFusedWarps = kFusedThreads / 32;
// resident CTAs per SM the register budget is sized for: 4 (64 registers) for
// SOC / RSOC tables, 2 (128) when the exponential-cone root solve is compiled in
constexpr int kFusedMinCtas = 4, kFusedMinCtasExp = 2;
constexpr int kSellC = 32;  // rows per slice
// elements per lane of the lane-group cone projections: a block of d elements takes
// g = d / kFusedEPL lanes (rounded up to a power of two), 32 / g blocks per warp
constexpr int kFusedEPL = 2;
// rows a thread updates at once in the step, their loads in flight together (2 spills
// registers under the 64-register budget and measured slower)
constexpr int kFusedRows = 1;

struct FusedTile {
  int32_t inst;    // instance
  int32_t o0, o1;  // instance-local row ordinals [o0, o1)
  int32_t ew;      // the first ew rows are elementwise (box / zero / nonneg)
  int32_t s0, s1;  // slices
  int32_t t0, t1;  // cone tasks
  int32_t x0, x1;  // exponential-cone records
  int32_t pad0, pad1;
};

struct FusedCsr {
  const FusedTile* tiles;
  int64_t ntiles;
  const int32_t* act;     // tiles of the iterating instances (NULL: every tile)
  const int64_t* n_act;
  const int64_t* sb;      // slice base (element offset of the slice's first column)
  const int32_t* sl;      // slice length (its longest row)
  const int16_t* so;      // per slice lane: tile-local row (-1: padding lane)
  const uint16_t* sc;     // SELL column (instance-local) of every stored element
  const int4* task;       // cone tasks {first record, records, lanes per group, 0}
  const int4* crec;       // cone records {merged start, length | RSOC << 30, cone, tile-local offset}
  const int4* xrec;       // exponential records {merged start, exp ordinal, tile-local offset, 0}
  RunTable rows, cols;    // row-side / column-side runs of every instance
  const int32_t* rloc;    // K * kMaxRuns: instance-local first row of each row run
  const int32_t* cloc;    // K * kMaxRuns: instance-local first column of each column run
  int32_t max_cols;       // staged elements (largest instance's column count)
  int32_t max_rows;       // largest tile's rows (products in shared memory)
  int32_t* sched;         // [0] next tile to hand out, [1] CTAs finished; both 0 between launches
};

// ---- fused ops.  In is what the update reads of row j (load), z(q, a, b)
// the value before the projection given the row's products (a, b: G'y for
// the primal step; G x, G x_lag for the dual one); Fin is what the store of
// the result reads (load_fin, or fin_of an In), fin(j, f, p, a, b, acc)
// stores the projection's result p and adds the control step's terms.

// FP32 bulk, primal: z = xa + dx_lag + tau_k (qa + G' dy_lag), dx = P(z) - xa;
// acc0 += (dx - dx_lag)^2
struct FusedPrimal32 {
  static constexpr int NACC = 1;
  const double* xa;
  float2* dxp;  // {dx, dx_lag}
  const double* qa;
  const double* ps;
  const uint8_t* mask;
  double sk = 0.0;
  struct In {
    double xa, qa;
    float dxl;
  };
  struct Fin {
    double xa;
    float dxl;
  };
  __device__ void begin(int64_t k) { sk = ps[k]; }
  __device__ In load(int64_t j) const { return {xa[j], qa[j], dxp[j].y}; }
  __device__ double z(const In& q, float a, float) const { return q.xa + (double)q.dxl + sk * (q.qa + (double)a); }
  __device__ Fin load_fin(int64_t j) const { return {xa[j], dxp[j].y}; }
  __device__ static Fin fin_of(const In& q) { return {q.xa, q.dxl}; }
  __device__ void fin(int64_t j, const Fin& f, double p, float, float, double* acc) const {
    const float d = (float)(p - f.xa);
    dxp[j].x = d;
    const double s = (double)d - (double)f.dxl;
    acc[0] += s * s;
  }
};

// FP32 bulk, dual: z = ya + dy_lag - sigma_k (ra + 2 G dx - G dx_lag), dy = P(z) - ya;
// acc0 += (dy - dy_lag)^2, acc1 += (dy - dy_lag)(G dx - G dx_lag)
struct FusedDual32 {
  static constexpr int NACC = 2;
  const double* ya;
  const float* dyl;
  const double* ra;
  float* dy;
  const double* ds;
  const uint8_t* mask;
  double sk = 0.0;
  struct In {
    double ya, ra;
    float dyl;
  };
  struct Fin {
    double ya;
    float dyl;
  };
  __device__ void begin(int64_t k) { sk = ds[k]; }
  __device__ In load(int64_t i) const { return {ya[i], ra[i], dyl[i]}; }
  __device__ double z(const In& q, float g, float gl) const {
    return q.ya + (double)q.dyl - sk * (q.ra + (2.0 * (double)g - (double)gl));
  }
  __device__ Fin load_fin(int64_t i) const { return {ya[i], dyl[i]}; }
  __device__ static Fin fin_of(const In& q) { return {q.ya, q.dyl}; }
  __device__ void fin(int64_t i, const Fin& f, double p, float g, float gl, double* acc) const {
    const float d = (float)(p - f.ya);
    dy[i] = d;
    const double s = (double)d - (double)f.dyl;
    acc[0] += s * s;
    acc[1] += s * ((double)g - (double)gl);
  }
};

// FP64, primal: x = P(x_lag + tau_k (G'y_lag - c)); acc0 += (x - x_lag)^2
struct FusedPrimal64 {
  static constexpr int NACC = 1;
  const double* xl;
  const double* c;
  double* out;
  const double* ps;
  const uint8_t* mask;
  double sk = 0.0;
  struct In {
    double xl, c;
  };
  struct Fin {
    double xl;
  };
  __device__ void begin(int64_t k) { sk = ps[k]; }
  __device__ In load(int64_t j) const { return {xl[j], c[j]}; }
  __device__ double z(const In& q, double a, double) const { return q.xl + sk * (a - q.c); }
  __device__ Fin load_fin(int64_t j) const { return {xl[j]}; }
  __device__ static Fin fin_of(const In& q) { return {q.xl}; }
  __device__ void fin(int64_t j, const Fin& f, double p, double, double, double* acc) const {
    out[j] = p;
    const double d = p - f.xl;
    acc[0] += d * d;
  }
};

// FP64, dual: y = P(y_lag - sigma_k (2 G x - G x_lag - h)); acc0 += (y - y_lag)^2,
// acc1 += (y - y_lag)(G x - G x_lag)
struct FusedDual64 {
  static constexpr int NACC = 2;
  const double* yl;
  const double* h;
  double* out;
  const double* ds;
  const uint8_t* mask;
  double sk = 0.0;
  struct In {
    double yl, h;
  };
  struct Fin {
    double yl;
  };
  __device__ void begin(int64_t k) { sk = ds[k]; }
  __device__ In load(int64_t i) const { return {yl[i], h[i]}; }
  __device__ double z(const In& q, double g, double gl) const { return q.yl - sk * ((2.0 * g - gl) - q.h); }
  __device__ Fin load_fin(int64_t i) const { return {yl[i]}; }
  __device__ static Fin fin_of(const In& q) { return {q.yl}; }
  __device__ void fin(int64_t i, const Fin& f, double p, double g, double gl, double* acc) const {
    out[i] = p;
    const double d = p - f.yl;
    acc[0] += d * d;
    acc[1] += d * (g - gl);
  }
};

// Asynchronous global -> shared copy of B = 4, 8 or 16 bytes (cp.async, cached
// in L1), both addresses aligned to B; cp_async_wait_all waits for this thread's
// copies (a barrier then makes every thread's visible).
template <int B>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
  static_assert(B == 4 || B == 8 || B == 16, "cp.async size");
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gmem), "n"(B) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// Shared memory before the products: the staged column segment, or (after the
// row pass) two doubles per tile row, whichever is larger.
template <class T, int NV>
__host__ __device__ inline size_t fused_stage_bytes(const FusedCsr& A) {
  const size_t a = sizeof(TileVal<T, NV>) * (size_t)(A.max_cols > 1 ? A.max_cols : 1);
  const size_t b = 2 * sizeof(double) * (size_t)(A.max_rows > 1 ? A.max_rows : 1);
  return ((a > b ? a : b) + 15) & ~size_t(15);
}

// The fused tile kernel.  T: matrix / product type; NV: 1 (G' y) or kPair /
// 2 (G applied to two vectors); EXP: compile the exponential-cone path.
// Dynamic shared memory: A.max_cols staged values, then the tile's products
// (1 or 2 per row, type T).
template <class T, int NV, class Op, bool EXP>
__global__ void __launch_bounds__(kFusedThreads, EXP ? kFusedMinCtasExp : kFusedMinCtas)
    fused_tile_kernel(FusedCsr A, const T* __restrict__ sv, const T* x0, const T* x1, Op op, ConeTable CT,
                      double* __restrict__ tpart, const int32_t* active) {
  if (active && !*active) return;
  using V = TileVal<T, NV>;
  constexpr int NP = NV == 1 ? 1 : 2;
  extern __shared__ __align__(16) unsigned char fused_smem[];
  const size_t stage = fused_stage_bytes<T, NV>(A);
  V* sx = reinterpret_cast<V*>(fused_smem);
  // after the row pass the staged segment is dead: the step keeps each row's value
  // before / after the projection (zs) and its cone scaling (ss) there
  double* zs = reinterpret_cast<double*>(fused_smem);
  double* ss = zs + A.max_rows;
  T* pr0 = reinterpret_cast<T*>(fused_smem + stage);
  T* pr1 = pr0 + A.max_rows;
  __shared__ int64_t run_row[kMaxRuns];
  __shared__ int32_t run_ord[kMaxRuns];
  __shared__ double red[Op::NACC][kFusedWarps];
  const int64_t nt = A.act ? *A.n_act : A.ntiles;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const double r2 = 0.7071067811865476;
  // Tiles are handed out one at a time from a counter, largest first (the order of
  // the active list), so a CTA that drew short tiles takes more of them.
  __shared__ int32_t s_next, s_slice, s_task;
  if (threadIdx.x == 0) s_next = atomicAdd(&A.sched[0], 1);
  __syncthreads();
  for (;;) {
    const int64_t q = s_next;
    if (q >= nt) break;
    const int64_t tid = A.act ? (int64_t)A.act[q] : q;
    const FusedTile tl = A.tiles[tid];
    const int64_t k = tl.inst;
    if (!op.mask[k]) {  // CTA-uniform: the instance does not iterate
      __syncthreads();  // every thread has read s_next
      if (threadIdx.x == 0) s_next = atomicAdd(&A.sched[0], 1);
      __syncthreads();
      continue;
    }
    if (threadIdx.x < kMaxRuns) {
      run_row[threadIdx.x] = A.rows.start[k * kMaxRuns + threadIdx.x];
      run_ord[threadIdx.x] = A.rloc[k * kMaxRuns + threadIdx.x];
    }
    if (threadIdx.x == 0) {  // the tile's slices and cone tasks are taken by the warps one at a time
      s_slice = 0;
      s_task = 0;
    }
    // the instance's column segment, copied to shared memory asynchronously (every copy
    // in flight at once, no registers held)
    for (int r = 0; r < kMaxRuns; ++r) {
      const int64_t s0 = A.cols.start[k * kMaxRuns + r], L = A.cols.len[k * kMaxRuns + r];
      V* dst = sx + A.cloc[k * kMaxRuns + r];
      if constexpr (NV == 2) {
        for (int64_t i = threadIdx.x; i < L; i += kFusedThreads) {
          cp_async<sizeof(T)>(&dst[i].x, x0 + s0 + i);
          cp_async<sizeof(T)>(&dst[i].y, x1 + s0 + i);
        }
      } else {
        const V* src = reinterpret_cast<const V*>(x0) + s0;
        for (int64_t i = threadIdx.x; i < L; i += kFusedThreads) cp_async<sizeof(V)>(dst + i, src + i);
      }
    }
    cp_async_wait_all();
    __syncthreads();
    // ---- the tile's rows, SELL-32: lane = row, one coalesced load per column ----
    for (;;) {
      int32_t si = 0;
      if (lane == 0) si = atomicAdd(&s_slice, 1);
      si = __shfl_sync(kFull, si, 0);
      if (si >= tl.s1 - tl.s0) break;
      const int64_t s = tl.s0 + si;
      const int64_t base = A.sb[s] + lane;
      const int32_t len = A.sl[s];
      const int32_t slot = A.so[s * kSellC + lane];
      T p0 = T(0), p1 = T(0);
      constexpr int U = sizeof(T) == 4 ? 16 : 4;
      for (int32_t j0 = 0; j0 < len; j0 += U) {
        T v[U];
        uint16_t c[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {  // every load of the chunk in flight together
          const bool ok = j0 + u < len;
          v[u] = ok ? sv[base + (int64_t)(j0 + u) * kSellC] : T(0);
          c[u] = ok ? A.sc[base + (int64_t)(j0 + u) * kSellC] : (uint16_t)0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const V xv = sx[c[u]];
          if constexpr (NV == 1) {
            p0 = fma(v[u], xv, p0);
          } else {
            p0 = fma(v[u], xv.x, p0);
            p1 = fma(v[u], xv.y, p1);
          }
        }
      }
      if (slot >= 0) {
        pr0[slot] = p0;
        if (NP == 2) pr1[slot] = p1;
      }
    }
    __syncthreads();
    // ---- the step of the tile's rows, in three passes over shared memory ----
    op.begin(k);
    double acc[Op::NACC];
#pragma unroll
    for (int a = 0; a < Op::NACC; ++a) acc[a] = 0.0;
    auto merged = [&](int64_t o) {  // instance-local ordinal -> merged index
      int r = 0;
      for (int t = 1; t < kMaxRuns; ++t)
        if (o >= run_ord[t]) r = t;
      return run_row[r] + (o - run_ord[r]);
    };
    const int nr = tl.o1 - tl.o0;
    // (a) every row's update in row order, kFusedRows rows per thread with their loads
    // issued together: elementwise rows are projected and stored here; a cone row's
    // value before the projection (and its scaling) goes to shared memory
    for (int i0 = threadIdx.x; i0 < nr; i0 += kFusedRows * kFusedThreads) {
      int64_t jj[kFusedRows];
      typename Op::In q[kFusedRows];
      double l[kFusedRows], h[kFusedRows];
      int32_t kd[kFusedRows];
#pragma unroll
      for (int u = 0; u < kFusedRows; ++u) {
        const int i = i0 + u * kFusedThreads;
        jj[u] = i < nr ? merged(tl.o0 + i) : -1;
        kd[u] = -1;
        l[u] = 1.0;
        h[u] = 1.0;
        if (jj[u] < 0) continue;
        q[u] = op.load(jj[u]);
        if (i < tl.ew) {
          kd[u] = CT.seg_kind[0];
          for (int g = 1; g < CT.nseg; ++g)
            if (jj[u] >= CT.seg_start[g]) kd[u] = CT.seg_kind[g];
          if (kd[u] == PK_BOX) {
            l[u] = CT.lo[jj[u]];
            h[u] = CT.hi[jj[u]];
          }
        } else if (CT.S) {
          l[u] = CT.S[jj[u]];
        }
      }
#pragma unroll
      for (int u = 0; u < kFusedRows; ++u) {
        const int i = i0 + u * kFusedThreads;
        if (jj[u] < 0) continue;
        const T a = pr0[i], b = NP == 2 ? pr1[i] : T(0);
        const double z = op.z(q[u], a, b);
        if (kd[u] >= 0) {
          const double p = kd[u] == PK_ZERO ? 0.0 : kd[u] == PK_NONNEG ? fmax(z, 0.0)
                           : kd[u] == PK_BOX ? fmin(fmax(z, l[u]), h[u]) : z;
          op.fin(jj[u], Op::fin_of(q[u]), p, a, b, acc);
        } else {
          zs[i] = z;
          ss[i] = l[u];
        }
      }
    }
    __syncthreads();
    // (b) SOC / RSOC blocks in lane groups of g lanes with kFusedEPL elements per lane,
    // on the values in shared memory; a warp takes the next task when it finishes one
    // (tasks cost different numbers of Newton steps), its descriptor in flight while the
    // current task is projected
    {
      const int32_t ntask = tl.t1 - tl.t0;
      int32_t t = 0;
      if (lane == 0) t = atomicAdd(&s_task, 1);
      t = __shfl_sync(kFull, t, 0);
      int4 tkn = make_int4(0, 0, 2, 0);
      if (t < ntask) tkn = A.task[tl.t0 + t];
      while (t < ntask) {
        const int4 tk = tkn;
        const int g = tk.z, gl = lane & (g - 1);
        const bool have = lane / g < tk.y;
        int4 rc = make_int4(0, 0, 0, 0);
        if (have) rc = A.crec[tk.x + lane / g];
        int32_t tn = 0;  // the warp's next task, its descriptor in flight during this one
        if (lane == 0) tn = atomicAdd(&s_task, 1);
        tn = __shfl_sync(kFull, tn, 0);
        if (tn < ntask) tkn = A.task[tl.t0 + tn];
        t = tn;
        const int d = have ? (rc.y & 0x3fffffff) : 0;
        const bool rsoc = have && (rc.y >> 30) != 0;
        const int l0 = rc.w;
        double* wsp = (have && CT.soc_ws) ? CT.soc_ws + rc.z : nullptr;
        const double wsv = (wsp && gl == 0) ? *wsp : __longlong_as_double(0x7ff8000000000000ll);
        // weights: S_0 / S_e (SOC), sqrt(S_0 S_1) / S_e for e >= 2 (RSOC); ss holds 1 when unscaled
        const double num = d > 0 ? (rsoc ? sqrt(ss[l0] * ss[l0 + 1]) : ss[l0]) : 1.0;
        double v[kFusedEPL], w[kFusedEPL];
        bool wne = false;
#pragma unroll
        for (int q = 0; q < kFusedEPL; ++q) {
          const int e = gl + g * q;
          v[q] = e < d ? zs[l0 + e] : 0.0;
          w[q] = (e < d && e >= (rsoc ? 2 : 1)) ? num / ss[l0 + e] : 1.0;
          wne |= w[q] != 1.0;
        }
        // the group is weighted when any of its elements has a weight != 1 (a vote)
        const unsigned gmask = g == 32 ? kFull : ((1u << g) - 1u) << (lane & ~(g - 1));
        const bool weighted = (__ballot_sync(kFull, wne) & gmask) != 0u;
        const bool any_rsoc = __any_sync(kFull, rsoc);
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
        if (any_rsoc) rotate();
        group_soc_multi<kFusedEPL>(v, w, d, weighted, g, wsv, wsp);
        if (any_rsoc) rotate();
#pragma unroll
        for (int q = 0; q < kFusedEPL; ++q) {
          const int e = gl + g * q;
          if (e < d) zs[l0 + e] = v[q];
        }
      }
    }
    if constexpr (EXP) {
      for (int64_t e = tl.x0 + threadIdx.x; e < tl.x1; e += kFusedThreads) {  // exponential cones
        const int4 xr = A.xrec[e];
        const int64_t kk = xr.y;
        const int li = xr.z;
        const bool first = kk < CT.exp_count;
        const int32_t kind = first ? CT.exp_kind : CT.dexp_kind;
        double zz[3];
#pragma unroll
        for (int u = 0; u < 3; ++u) zz[u] = zs[li + u];
        double S0 = 1.0, S1 = 1.0, S2 = 1.0;
        if (CT.S) {
          S0 = ss[li];
          S1 = ss[li + 1];
          S2 = ss[li + 2];
        }
        double* ws = CT.rho_ws ? CT.rho_ws + kk : nullptr;
        if (kind == PK_EXP) proj_exp_scaled_dev(zz[0], zz[1], zz[2], S0, S1, S2, ws);
        else proj_dexp_scaled_dev(zz[0], zz[1], zz[2], S0, S1, S2, ws);
#pragma unroll
        for (int u = 0; u < 3; ++u) zs[li + u] = zz[u];
      }
    }
    __syncthreads();
    // the next tile, published by the barrier of the partial sums below (every thread
    // read this tile's index at the top of the loop, several barriers ago)
    if (threadIdx.x == 0) s_next = atomicAdd(&A.sched[0], 1);
    // (c) the cone rows' results, stored in row order with the control step's terms
    for (int i0 = tl.ew + threadIdx.x; i0 < nr; i0 += kFusedRows * kFusedThreads) {
      int64_t jj[kFusedRows];
      typename Op::Fin f[kFusedRows];
#pragma unroll
      for (int u = 0; u < kFusedRows; ++u) {
        const int i = i0 + u * kFusedThreads;
        jj[u] = i < nr ? merged(tl.o0 + i) : -1;
        if (jj[u] >= 0) f[u] = op.load_fin(jj[u]);
      }
#pragma unroll
      for (int u = 0; u < kFusedRows; ++u) {
        const int i = i0 + u * kFusedThreads;
        if (jj[u] < 0) continue;
        const T a = pr0[i], b = NP == 2 ? pr1[i] : T(0);
        op.fin(jj[u], f[u], zs[i], a, b, acc);
      }
    }
    // ---- the tile's partial sums, in a fixed order ----
#pragma unroll
    for (int a = 0; a < Op::NACC; ++a) {
      double v = acc[a];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
      if (lane == 0) red[a][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < Op::NACC) {
      double v = red[threadIdx.x][0];
      for (int w = 1; w < kFusedWarps; ++w) v += red[threadIdx.x][w];
      tpart[tid * Op::NACC + threadIdx.x] = v;
    }
    // no barrier here: the next tile's first writes to shared memory (run tables, staged
    // segment) touch nothing read after the barrier above, and red is rewritten only
    // after the next tile's own barriers
  }
  // the last CTA to finish resets the counters for the next launch (every other CTA
  // is past its last read of them)
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&A.sched[1], 1) == (int32_t)gridDim.x - 1) {
      A.sched[0] = 0;
      A.sched[1] = 0;
      __threadfence();
    }
  }
}

// Builds the SELL arrays on the device: slice s, lane l holds merged row
// srow[s * 32 + l] (-1: padding); its nonzeros go to sv / sc[sb[s] + j * 32 + l]
// for j < the row's length, zeros (column 0) to the slice's length.
template <class T>
__global__ void sell_fill_kernel(int64_t nslices, const int64_t* __restrict__ sb, const int32_t* __restrict__ sl,
                                 const int32_t* __restrict__ srow, const int32_t* __restrict__ rp,
                                 const T* __restrict__ vals, const uint16_t* __restrict__ cl, T* __restrict__ sv,
                                 uint16_t* __restrict__ sc) {
  const int64_t total = nslices * kSellC;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += stride) {
    const int64_t s = q / kSellC;
    const int l = (int)(q % kSellC);
    const int32_t r = srow[q];
    const int64_t b = sb[s] + l;
    const int32_t L = sl[s];
    const int32_t e0 = r >= 0 ? rp[r] : 0, n = r >= 0 ? rp[r + 1] - rp[r] : 0;
    for (int32_t j = 0; j < L; ++j) {
      const bool ok = j < n;
      sv[b + (int64_t)j * kSellC] = ok ? vals[e0 + j] : T(0);
      sc[b + (int64_t)j * kSellC] = ok ? cl[e0 + j] : (uint16_t)0;
    }
  }
}

template <class T, int NV>
inline size_t fused_smem_bytes(const FusedCsr& A) {
  return fused_stage_bytes<T, NV>(A) + sizeof(T) * (NV == 1 ? 1 : 2) * (size_t)std::max(A.max_rows, 1);
}

// Raise the kernel's dynamic shared memory limit to what A needs (per device,
// only ever growing: graphs captured with larger tiles stay launchable).
template <class T, int NV, class Op, bool EXP>
inline void fused_prepare(const FusedCsr& A) {
  static std::mutex mu;
  static std::map<int, size_t> set;
  int dev = 0;
  PDCS_CUDA(cudaGetDevice(&dev));
  const size_t need = fused_smem_bytes<T, NV>(A);
  std::lock_guard<std::mutex> lock(mu);
  if (need <= set[dev]) return;
  PDCS_CUDA(cudaFuncSetAttribute(fused_tile_kernel<T, NV, Op, EXP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)need));
  set[dev] = need;
}

template <class T, int NV, class Op>
inline void launch_fused(const FusedCsr& A, int grid, const T* sv, const std::type_identity_t<T>* x0,
                         const std::type_identity_t<T>* x1, const Op& op, const ConeTable& CT, double* tpart,
                         const int32_t* active, cudaStream_t s) {
  const size_t smem = fused_smem_bytes<T, NV>(A);
  if (CT.exp_count + CT.dexp_count > 0)
    fused_tile_kernel<T, NV, Op, true><<<grid, kFusedThreads, smem, s>>>(A, sv, x0, x1, op, CT, tpart, active);
  else
    fused_tile_kernel<T, NV, Op, false><<<grid, kFusedThreads, smem, s>>>(A, sv, x0, x1, op, CT, tpart, active);
}

}  // namespace pdcs
