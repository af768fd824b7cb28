// pdcs_solver.cu -- B200-native restarted, diagonally preconditioned,
// adaptive-step PDHG for PDCS conic programs, behind the C ABI of pdcs.h.
//
// Host control mirrors the reference's aggressive main loop
// (src/pdcs_gpu/rpdhg_alg_gpu_gen_scaling.jl:770-895).  The inner loop runs on
// the device: PDHG attempts are captured in CUDA graphs and the accept/retry
// decision, step sizes and the reflected averaging are computed by kernels on a
// device-resident state, so the host only intervenes at the reference's
// checkpoints (iter % check_terminate_freq, restart checks, artificial restarts).
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/pdcs.h"
#include "pdcs_fp32.cuh"
#include "pdcs_kernels.cuh"
#include "pdcs_preprocess.cuh"

namespace pdcs {

// ===========================================================================
// Kernels with a single instantiation
// ===========================================================================

__global__ void finalize_partials_kernel2(const double* __restrict__ partials, int nblocks, int nacc,
                                          uint32_t maxmask, double* __restrict__ out) {
  const int k = blockIdx.x;
  if (k >= nacc) return;
  const bool mx = (maxmask >> k) & 1u;
  double v = 0.0;
  for (int i = threadIdx.x; i < nblocks; i += blockDim.x) {
    double p = partials[(int64_t)k * nblocks + i];
    v = mx ? fmax(v, p) : v + p;
  }
  __shared__ double sh[kThreads];
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] = mx ? fmax(sh[threadIdx.x], sh[threadIdx.x + s]) : sh[threadIdx.x] + sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[k] = sh[0];
}

// DotSpec kinds
enum DotKind : int32_t { DK_DOT = 0, DK_MAXABS = 1, DK_SUMABS = 2, DK_DIFF2 = 3 };

__global__ void __launch_bounds__(kThreads) dots_kernel(DotSpec spec, double* partials) {
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  const int64_t stride = (int64_t)gridDim.x * kThreads;
  for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < spec.len; i += stride) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (k >= spec.count) break;
      double a = spec.a[k][i];
      if (spec.sa[k]) a /= spec.sa[k][i];
      switch (spec.kind[k]) {
        case DK_DOT: acc[k] = fma(a, spec.b[k] ? spec.b[k][i] : a, acc[k]); break;
        case DK_MAXABS: acc[k] = fmax(acc[k], fabs(a)); break;
        case DK_SUMABS: acc[k] += fabs(a); break;
        case DK_DIFF2: { double d = a - spec.b[k][i]; acc[k] = fma(d, d, acc[k]); } break;
      }
    }
  }
  __shared__ double sh[4][kWarps];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    double v = acc[k];
    const bool mx = spec.kind[k] == DK_MAXABS;
    for (int o = 16; o > 0; o >>= 1) v = mx ? fmax(v, __shfl_down_sync(kFull, v, o)) : v + __shfl_down_sync(kFull, v, o);
    if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    const int k = threadIdx.x;
    const bool mx = spec.kind[k] == DK_MAXABS;
    double v = sh[k][0];
    for (int w = 1; w < kWarps; ++w) v = mx ? fmax(v, sh[k][w]) : v + sh[k][w];
    partials[(int64_t)k * gridDim.x + blockIdx.x] = v;
  }
}

__global__ void __launch_bounds__(kThreads) reflect_kernel(PdhgState* st, double* __restrict__ x,
                                                           double* __restrict__ xl, double* __restrict__ xm,
                                                           int64_t n, double* __restrict__ y, double* __restrict__ yl,
                                                           double* __restrict__ ym, int64_t m) {
  if (!st->do_reflect) return;  // set by this attempt's control step, cleared by the next attempt's first kernel
  const double tmp = st->refl_tmp, inv = st->refl_inv, e = st->refl_extra, eta = st->refl_eta, cum = st->refl_cum;
  const double wsum = cum + eta;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t L = n > m ? n : m;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < L; i += stride) {
    if (i < n) {
      double xv = x[i];
      double xn = tmp * ((1.0 + e) * xv - e * xl[i]) + inv * xv;
      xm[i] = (xm[i] * cum + xn * eta) / wsum;
      x[i] = xn;
      xl[i] = xn;
    }
    if (i < m) {
      double yv = y[i];
      double yn = tmp * ((1.0 + e) * yv - e * yl[i]) + inv * yv;
      ym[i] = (ym[i] * cum + yn * eta) / wsum;
      y[i] = yn;
      yl[i] = yn;
    }
  }
}

// ---------------------------------------------------------------------------
// Merge-path CSR SpMV (Merrill & Garland, "Merge-based parallel sparse
// matrix-vector multiplication", SC'16): the m row ends and the nnz nonzeros
// form m + nnz merge items split evenly over CTAs (kMergeItems per CTA, 8 per
// thread), so the work per CTA is independent of the row-length distribution.
// Every row end is consumed by exactly one thread, which writes y[row]; the
// partial sum of a row that continues past a thread's items is combined
// inside the CTA, and the partial of a row that continues past the CTA
// becomes the CTA's carry (carry_row / carry_val, one entry per CTA), added
// in CTA order by spmv_merge_fixup_kernel.
// ---------------------------------------------------------------------------
constexpr int kMergeIPT = 8;
constexpr int kMergeItems = kThreads * kMergeIPT;

__device__ inline void merge_path_search(int64_t diag, const int32_t* __restrict__ row_end, int64_t nrows,
                                         int64_t nnz, int64_t* row, int64_t* k) {
  int64_t lo = diag - nnz > 0 ? diag - nnz : 0;
  int64_t hi = diag < nrows ? diag : nrows;
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if ((int64_t)row_end[mid] <= diag - mid - 1) lo = mid + 1;
    else hi = mid;
  }
  *row = lo;
  *k = diag - lo;
}

__global__ void __launch_bounds__(kThreads) spmv_merge_kernel(int64_t m, int64_t nnz, const int32_t* __restrict__ rp,
                                                              const int32_t* __restrict__ ci,
                                                              const double* __restrict__ v,
                                                              const double* __restrict__ x, double* __restrict__ y,
                                                              int32_t* __restrict__ carry_row,
                                                              double* __restrict__ carry_val) {
  const int64_t total = m + nnz;
  const int64_t d0 = (int64_t)blockIdx.x * kMergeItems;
  const int64_t d1 = d0 + kMergeItems < total ? d0 + kMergeItems : total;
  const int32_t* row_end = rp + 1;
  __shared__ int64_t s_r0, s_r1;
  __shared__ int64_t s_row[kThreads];
  __shared__ double s_val[kThreads];
  if (threadIdx.x == 0) {
    int64_t kk;
    merge_path_search(d0, row_end, m, nnz, &s_r0, &kk);
    merge_path_search(d1, row_end, m, nnz, &s_r1, &kk);
  }
  __syncthreads();
  const int nvalid = (int)((d1 - d0 + kMergeIPT - 1) / kMergeIPT);
  const int t = threadIdx.x;
  const int64_t dt = d0 + (int64_t)t * kMergeIPT;
  int64_t row = -1;
  double sum = 0.0;
  if (t < nvalid) {
    const int64_t dte = dt + kMergeIPT < d1 ? dt + kMergeIPT : d1;
    // search only inside this CTA's row range [s_r0, s_r1]
    int64_t lo = dt - nnz > s_r0 ? dt - nnz : s_r0;
    int64_t hi = dt < s_r1 ? dt : s_r1;
    while (lo < hi) {
      int64_t mid = (lo + hi) >> 1;
      if ((int64_t)row_end[mid] <= dt - mid - 1) lo = mid + 1;
      else hi = mid;
    }
    row = lo;
    int64_t k = dt - lo;
    for (int64_t it = dt; it < dte; ++it) {
      if (row < m && k < (int64_t)row_end[row]) {
        sum = fma(v[k], x[ci[k]], sum);
        ++k;
      } else {
        y[row] = sum;  // this thread consumed the end of `row`
        sum = 0.0;
        ++row;
      }
    }
    if (row >= m) row = -1;  // finished every row: nothing carried
  }
  s_row[t] = row;
  s_val[t] = sum;
  __syncthreads();
  // Threads t..u-1 that all stop inside row r form a run.  If thread u < nvalid
  // exists it started inside row r and moved past it, so it consumed row r's
  // end and already wrote y[r]; otherwise row r continues into the next CTA.
  const int64_t r = s_row[t];
  if (t < nvalid && r >= 0 && (t == 0 || s_row[t - 1] != r)) {
    double acc = 0.0;
    int u = t;
    while (u < nvalid && s_row[u] == r) acc += s_val[u++];
    if (u < nvalid) {
      y[r] += acc;
    } else {
      carry_row[blockIdx.x] = (int32_t)r;
      carry_val[blockIdx.x] = acc;
    }
  }
  if (t == 0 && s_row[nvalid - 1] < 0) {  // no row continues past this CTA
    carry_row[blockIdx.x] = -1;
    carry_val[blockIdx.x] = 0.0;
  }
}

// y[carry_row[c]] += carry_val[c], summing consecutive carries of one row in CTA order
__global__ void spmv_merge_fixup_kernel(int64_t nctas, const int32_t* __restrict__ carry_row,
                                        const double* __restrict__ carry_val, double* __restrict__ y) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nctas; c += stride) {
    const int32_t r = carry_row[c];
    if (r < 0 || (c > 0 && carry_row[c - 1] == r)) continue;
    double acc = 0.0;
    for (int64_t u = c; u < nctas && carry_row[u] == r; ++u) acc += carry_val[u];
    y[r] += acc;
  }
}

// out = a*u + b*v (u, v may alias out)
__global__ void axpby_kernel(double* out, double a, const double* u, double b, const double* v, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    out[i] = a * u[i] + (v ? b * v[i] : 0.0);
}
// out = u / d
__global__ void div_kernel(double* out, const double* u, const double* d, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) out[i] = u[i] / d[i];
}

// standalone projection entry (pdcs_block_proj): one block per CTA-warp
__global__ void __launch_bounds__(kThreads) block_proj_kernel(double* arr, const double* bl, const double* bu,
                                                              const double* S, const int64_t* head,
                                                              const int64_t* ns, int64_t nblk,
                                                              const int64_t* code) {
  const int lane = threadIdx.x & 31;
  const int64_t wid = ((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5;
  const int64_t wstride = ((int64_t)gridDim.x * kThreads) >> 5;
  const double r2 = 0.7071067811865476;
  for (int64_t b = wid; b < nblk; b += wstride) {
    const int64_t st = head[b], d = ns[b];
    const int64_t c = code[b];
    double* p = arr + st;
    switch (c) {
      case 0: case 1: break;
      case 2: for (int64_t i = lane; i < d; i += 32) p[i] = 0.0; break;
      case 3: case 4: for (int64_t i = lane; i < d; i += 32) p[i] = fmax(p[i], 0.0); break;
      case 17: case 18: case 19:
        for (int64_t i = lane; i < d; i += 32) p[i] = fmin(fmax(p[i], bl[st + i]), bu[st + i]);
        break;
      case 5: case 7: case 20: case 21:
        warp_soc_mem(p, d, [](int64_t) { return 1.0; }, false);
        break;
      case 6: case 22: {
        const double* Sb = S + st;
        warp_soc_mem(p, d, [&](int64_t i) { return Sb[0] / Sb[i]; }, true);
      } break;
      case 8: case 10: case 23: case 24: case 9: case 25: {
        const bool sc = (c == 9 || c == 25);
        const double* Sb = sc ? S + st : nullptr;
        if (d >= 3) {
          if (lane == 0) {
            double p0 = p[0], q0 = p[1];
            p[0] = (p0 + q0) * r2;
            p[1] = (p0 - q0) * r2;
          }
          __syncwarp();
          double g = sc ? sqrt(Sb[0] * Sb[1]) : 1.0;
          warp_soc_mem(p, d, [&](int64_t i) { return (i == 1 || !sc) ? 1.0 : g / Sb[i]; }, sc);
          __syncwarp();
          if (lane == 0) {
            double a0 = p[0], b0 = p[1];
            p[0] = (a0 + b0) * r2;
            p[1] = (a0 - b0) * r2;
          }
        } else {
          for (int64_t i = lane; i < d; i += 32) p[i] = fmax(p[i], 0.0);
        }
      } break;
      case 11: case 16: case 28: case 12: case 29:
        if (lane == 0 && d == 3) {
          double Sr = 1.0, Ss = 1.0, St = 1.0;
          if (c == 12 || c == 29) { Sr = S[st]; Ss = S[st + 1]; St = S[st + 2]; }
          proj_dexp_scaled_dev(p[0], p[1], p[2], Sr, Ss, St);
        }
        break;
      case 13: case 14: case 26: case 15: case 27:
        if (lane == 0 && d == 3) {
          double Sr = 1.0, Ss = 1.0, St = 1.0;
          if (c == 15 || c == 27) { Sr = S[st]; Ss = S[st + 1]; St = S[st + 2]; }
          proj_exp_scaled_dev(p[0], p[1], p[2], Sr, Ss, St);
        }
        break;
      default: break;
    }
    __syncwarp();
  }
}

// ===========================================================================
// Host side
// ===========================================================================

struct CudaError : std::runtime_error {
  explicit CudaError(const std::string& s) : std::runtime_error(s) {}
};
#define PDCS_CUDA(call)                                                                         \
  do {                                                                                          \
    cudaError_t e__ = (call);                                                                   \
    if (e__ != cudaSuccess)                                                                     \
      throw CudaError(std::string(#call) + ": " + cudaGetErrorString(e__));                    \
  } while (0)

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// One stream-ordered memory pool per device, owned by the library: a solve's
// workspace returns to it at the end and the next solve on that device reuses
// it without driver allocations (cudaMalloc / cudaFree synchronise the device).
// Up to kPoolKeep bytes stay cached across synchronisations.
constexpr uint64_t kPoolKeep = 8ull << 30;

static cudaMemPool_t library_pool() {
  static std::mutex mu;
  static std::vector<cudaMemPool_t> pools;
  int dev = 0;
  PDCS_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if ((int)pools.size() <= dev) pools.resize(dev + 1, nullptr);
  if (!pools[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    PDCS_CUDA(cudaMemPoolCreate(&pool, &props));
    uint64_t keep = kPoolKeep;
    PDCS_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    pools[dev] = pool;
  }
  return pools[dev];
}

// Device workspace of one solve, allocated in stream order on the solve's stream.
struct Arena {
  std::vector<void*> ptrs;
  cudaStream_t s = nullptr;
  cudaMemPool_t pool = nullptr;
  void bind(cudaStream_t stream) {
    s = stream;
    pool = library_pool();
  }
  template <class T>
  T* alloc(size_t count) {
    void* p = nullptr;
    PDCS_CUDA(cudaMallocFromPoolAsync(&p, std::max<size_t>(count, 1) * sizeof(T), pool, s));
    ptrs.push_back(p);
    return static_cast<T*>(p);
  }
  void release() {
    for (void* p : ptrs) cudaFreeAsync(p, s);
    ptrs.clear();
  }
  void drop(const void* p) {
    for (size_t i = 0; i < ptrs.size(); ++i)
      if (ptrs[i] == p) {
        cudaFreeAsync(ptrs[i], s);
        ptrs.erase(ptrs.begin() + i);
        return;
      }
  }
  ~Arena() { release(); }
};

struct Converge {
  double pobj = 1e30, dobj = 1e30, abs_gap = 1e30, rel_gap = 1e30;
  double linf_rel_p = 1e30, linf_rel_d = 1e30, l2_rel_p = 1e30, l2_rel_d = 1e30;
  double linf_abs_p = 1e30, linf_abs_d = 1e30, l2_abs_p = 1e30, l2_abs_d = 1e30;
  int status = PDCS_EXIT_CONTINUE;
};

struct Infea {
  double max_primal_ray_inf = 1e30, primal_ray_obj = 1e30, max_dual_ray_inf = 1e30, dual_ray_obj = 1e30;
  double primal_ray_norm = 0, dual_ray_norm = 0;
  std::vector<double> ptrend, dtrend;
  int status = PDCS_EXIT_CONTINUE;
};

class Solver {
 public:
  // true when a part-D barrier of the last solve gave up (its projection is invalid)
  bool huge_failed() {
    if (!huge_err_) return false;
    int32_t e = 0;
    PDCS_CUDA(cudaMemcpyAsync(&e, huge_err_, sizeof(int32_t), cudaMemcpyDeviceToHost, s_));
    PDCS_CUDA(cudaStreamSynchronize(s_));
    return e != 0;
  }
  Solver(const pdcs_problem* p, const pdcs_options* o) : P(*p), O(*o) {}
  virtual ~Solver() {
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    if (graph_) cudaGraphDestroy(graph_);
    if (host_state_) cudaFreeHost(host_state_);
    if (host_red_) cudaFreeHost(host_red_);
    A.release();  // back to the pool, in order on s_
    if (own_stream_) cudaStreamDestroy(s_);
  }
  int run(pdcs_result* res);
  int validate_only() { return validate(); }

 protected:
  pdcs_problem P;
  pdcs_options O;
  Arena A;
  cudaStream_t s_ = nullptr;
  bool own_stream_ = false;
  int64_t n_ = 0, m_ = 0, nb_ = 0, nnz_ = 0;
  // device data
  CsrDev G_{}, Gt_{};
  double *c_s = nullptr, *c_raw = nullptr, *h_s = nullptr, *h_raw = nullptr, *Dr = nullptr, *Dl = nullptr;
  double *bl_s = nullptr, *bu_s = nullptr, *lam_l = nullptr, *lam_u = nullptr, *bl_fin = nullptr, *bu_fin = nullptr;
  double *x = nullptr, *xl = nullptr, *xm = nullptr, *aty = nullptr, *x0 = nullptr, *x0l = nullptr, *xbest = nullptr;
  double *y = nullptr, *yl = nullptr, *ym = nullptr, *gx = nullptr, *gxl = nullptr, *y0 = nullptr, *y0l = nullptr,
         *ybest = nullptr;
  double *tn[6] = {}, *tm[6] = {};
  double *xds_ = nullptr, *yds_ = nullptr;  // iterates at the start of an outer iteration (omega update)
  // FP32-bulk mode (precision 1): FP32 matrices and deltas, FP64 anchors and averages
  bool fp32_ = false;
  CsrT<float> G32_{}, Gt32_{};
  float2* dxp32_ = nullptr;  // {dx, dxl} pairs
  float *dy32_ = nullptr, *dyl32_ = nullptr;
  float *aty32_ = nullptr, *gx32_ = nullptr, *gxl32_ = nullptr;
  double *xa_ = nullptr, *ya_ = nullptr, *qa_ = nullptr, *ra_ = nullptr, *dxm_ = nullptr, *dym_ = nullptr;
  // differentiable mode: the unscaled data the solution-map adjoint works on
  CsrDev Graw_{}, Gtraw_{};
  double *bl_raw_ = nullptr, *bu_raw_ = nullptr;
  double *part_x = nullptr, *part_y = nullptr, *part_r = nullptr, *red_out = nullptr;
  double *part_a = nullptr, *part_b = nullptr;  // partials of host-driven (non-graph) reductions
  PdhgState* st_dev = nullptr;
  PdhgState* host_state_ = nullptr;
  double* host_red_ = nullptr;
  // part D of the update kernels (huge SOC / RSOC blocks): barrier state, the
  // flag a CTA sets when it gave up waiting, partial sums
  unsigned* huge_bar_ = nullptr;
  int32_t* huge_err_ = nullptr;
  double* huge_red_ = nullptr;

  ConeTable XI{}, YI{}, CON{}, SLK{};
  int grid_reflect_ = 1, grid_vec_n_ = 1, grid_vec_m_ = 1;
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t graph_exec_ = nullptr;
  int attempts_per_graph_ = 32;
  double ginf_ = 0.0, hNrm1 = 0, hNrmInf = 0, cNrm1 = 0, cNrmInf = 0;
  // algorithm state (host mirror of Solution / PDHGCLPInfo)
  PdhgState S{};
  Converge ci[2];
  Infea ii[2];
  int exit_code_ = PDCS_EXIT_CONTINUE;
  int returned_seq_ = 0;
  double pobj_ = 1e30, dobj_ = 1e30;
  double max_kkt_ = 1e30, min_kkt_ = 1e30;
  double pres_best_ = 1e30, dres_best_ = 1e30;
  double ndg_[2] = {1e30, 1e30}, ndg_thr_ = 0, ndg_r_ = 1e30, kkt_err_[2] = {1e30, 1e30}, kkt_thr_ = 0;
  bool dgap_flag_ = true;
  double bs_t0_ = 1.0;
  int64_t restart_used_ = 0, check_count_ = 0;
  double t_start_ = 0;
  int64_t kernels_ = 0, graphs_ = 0, probes_ = 0;
  double t_iter_ = 0, t_exit_ = 0, t_restart_ = 0;
  struct Timer {
    double& acc;
    double t0;
    explicit Timer(double& a) : acc(a), t0(now_s()) {}
    ~Timer() { acc += now_s() - t0; }
  };

  // ---- setup ----
  int validate();
  void setup();
  // G's CSR arrays onto the device (the batch assembles its merged matrix there)
  virtual void upload_matrix(int32_t* g_rp, int32_t* g_ci, double* g_v) {
    const cudaMemcpyKind kind = P.on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    PDCS_CUDA(cudaMemcpyAsync(g_rp, P.G_rowptr, sizeof(int32_t) * (m_ + 1), kind, s_));
    if (nnz_) {
      PDCS_CUDA(cudaMemcpyAsync(g_ci, P.G_colind, sizeof(int32_t) * nnz_, kind, s_));
      PDCS_CUDA(cudaMemcpyAsync(g_v, P.G_val, sizeof(double) * nnz_, kind, s_));
    }
  }
  // verbose: wall time of each setup phase, the stream synchronised at every mark
  double phase_t_ = 0.0;
  void phase(const char* name) {
    if (!O.verbose) return;
    PDCS_CUDA(cudaStreamSynchronize(s_));
    const double t = now_s();
    if (phase_t_ > 0.0) std::printf("[pdcs_b200 setup] %-28s %8.3f ms\n", name, 1e3 * (t - phase_t_));
    phase_t_ = t;
  }
  void build_bins(const std::vector<int32_t>& rp, int64_t rows, int64_t cols, const int32_t* d_rp,
                  const int32_t* d_ci, const double* d_v, CsrDev& D, const int32_t* row_inst, int lane_nnz);
  int tune_bins(const std::vector<int32_t>& rp, int64_t rows, int64_t cols, const int32_t* d_rp, const int32_t* d_ci,
                const double* d_v, CsrDev& D, const int32_t* row_inst, const double* xin, double* yout,
                const float* v32 = nullptr);
  float* gv32_ = nullptr;  // FP32 values of G and G' (FP32-bulk mode), converted before the schedules are tuned
  float* tv32_ = nullptr;
  int lane_G_ = 4, lane_Gt_ = 4;  // SpMV schedules in use (nonzeros per lane)
  // split-row workspaces (chunk partials, row counters) per matrix, keyed on its row pointers
  std::map<const int32_t*, std::pair<double*, unsigned*>> split_ws_;
  // instance of each row of G and of G' (batched solver; NULL: one instance)
  const int32_t* inst_of_y_ = nullptr;
  const int32_t* inst_of_x_ = nullptr;
  int warp_grid(int64_t rows) const {
    return (int)std::max<int64_t>(1, std::min<int64_t>((rows * 32 + kThreads - 1) / kThreads, 148 * 16));
  }
  void build_tables(const std::vector<int64_t>& soc_x, const std::vector<int64_t>& rsoc_x,
                    const std::vector<int64_t>& socG, const std::vector<int64_t>& rsocG);
  void size_table(ConeTable& T);
  void capture_graph();
  // ---- device helpers ----
  void spmv(const CsrDev& M, const double* xin, double* yout) {
    launch_spmv<1>(M, xin, nullptr, yout, nullptr, nullptr, s_);
    kernels_++;
  }
  // rows of the instances with mask[k] != 0 only (batched solver)
  void spmv_masked(const CsrDev& M, const double* xin, double* yout, const uint8_t* mask) {
    launch_spmv<1, true>(M, xin, nullptr, yout, nullptr, nullptr, s_, nullptr, mask);
    kernels_++;
  }
  void axpby(double* out, double a, const double* u, double b, const double* v, int64_t len) {
    axpby_kernel<<<grid_for(len), kThreads, 0, s_>>>(out, a, u, b, v, len);
    kernels_++;
  }
  void copy(double* dst, const double* src, int64_t len) {
    PDCS_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * len, cudaMemcpyDeviceToDevice, s_));
  }
  int grid_for(int64_t len) const { return (int)std::max<int64_t>(1, std::min<int64_t>((len + kThreads - 1) / kThreads, 148 * 8)); }
  template <class Op>
  void update_project(const Op& op, const ConeTable& T, double* partials) {
    launch_update_project(op, T, partials, nullptr, s_);
    kernels_++;
  }
  // reduce partials of the last kernel to host values
  void finalize(const double* partials, int nblocks, int nacc, uint32_t maxmask, double* out_host) {
    finalize_partials_kernel2<<<nacc, kThreads, 0, s_>>>(partials, nblocks, nacc, maxmask, red_out);
    kernels_++;
    PDCS_CUDA(cudaMemcpyAsync(host_red_, red_out, sizeof(double) * nacc, cudaMemcpyDeviceToHost, s_));
    PDCS_CUDA(cudaStreamSynchronize(s_));
    for (int k = 0; k < nacc; ++k) out_host[k] = host_red_[k];
  }
  void dots(DotSpec spec, double* out_host) {
    int g = grid_for(spec.len);
    for (int k = spec.count; k < 4; ++k) {
      spec.a[k] = spec.a[0];
      spec.b[k] = nullptr;
      spec.sa[k] = nullptr;
      spec.kind[k] = DK_DOT;
    }
    dots_kernel<<<g, kThreads, 0, s_>>>(spec, part_r);
    kernels_++;
    uint32_t mask = 0;
    for (int k = 0; k < 4; ++k)
      if (spec.kind[k] == DK_MAXABS) mask |= 1u << k;
    double tmp[4];
    finalize(part_r, g, 4, mask, tmp);
    for (int k = 0; k < spec.count; ++k) out_host[k] = tmp[k];
  }
  double nrm2(const double* a, int64_t len) {
    DotSpec d{};
    d.a[0] = a;
    d.kind[0] = DK_DOT;
    d.count = 1;
    d.len = len;
    double v;
    dots(d, &v);
    return std::sqrt(v);
  }
  // ---- asynchronous reductions: results land in slots of red_out, fetched together ----
  void finalize_async(const double* partials, int nblocks, int nacc, uint32_t maxmask, int slot) {
    finalize_partials_kernel2<<<nacc, kThreads, 0, s_>>>(partials, nblocks, nacc, maxmask, red_out + slot);
    kernels_++;
  }
  void dots_async(DotSpec spec, double* partials, int slot) {
    int g = grid_for(spec.len);
    uint32_t mask = 0;
    for (int k = spec.count; k < 4; ++k) {
      spec.a[k] = spec.a[0];
      spec.b[k] = nullptr;
      spec.sa[k] = nullptr;
      spec.kind[k] = DK_DOT;
    }
    for (int k = 0; k < 4; ++k)
      if (spec.kind[k] == DK_MAXABS) mask |= 1u << k;
    dots_kernel<<<g, kThreads, 0, s_>>>(spec, partials);
    kernels_++;
    finalize_async(partials, g, spec.count, mask, slot);
  }
  const double* fetch(int count) {
    PDCS_CUDA(cudaMemcpyAsync(host_red_, red_out, sizeof(double) * count, cudaMemcpyDeviceToHost, s_));
    PDCS_CUDA(cudaStreamSynchronize(s_));
    return host_red_;
  }
  template <class Op>
  int launch_project(const Op& op, const ConeTable& T, double* partials) {
    update_project(op, T, partials);
    return table_grid(T);
  }

  void push_state() {
    // synchronous w.r.t. the pinned staging buffer, which the next push reuses
    *host_state_ = S;
    PDCS_CUDA(cudaMemcpyAsync(st_dev, host_state_, sizeof(PdhgState), cudaMemcpyHostToDevice, s_));
    PDCS_CUDA(cudaStreamSynchronize(s_));
  }
  void pull_state() {
    PDCS_CUDA(cudaMemcpyAsync(host_state_, st_dev, sizeof(PdhgState), cudaMemcpyDeviceToHost, s_));
    PDCS_CUDA(cudaStreamSynchronize(s_));
    S = *host_state_;
  }
  // ---- algorithm ----
  double decay(double mk) const { return std::min(0.9 + 0.1 * std::log10(mk * 1e5), 1.0); }
  void converge_info(const double* xs, const double* ys, Converge& C, double* gxs, double* atys);
  void exit_check();
  void check_termination();
  double mnorm(const double* dx, const double* dy, double ta, double si);
  double binary_search(double r, const double* px, const double* py, double ta, double si);
  double kkt_error(const Converge& C) const {
    return std::sqrt(S.omega * S.omega * C.l2_abs_p * C.l2_abs_p + C.l2_abs_d * C.l2_abs_d / (S.omega * S.omega) +
                     C.abs_gap * C.abs_gap);
  }
  void restart_threshold(bool dgap);
  bool restart_check(bool dgap);
  double init_omega() {
    double hn = nrm2(h_s, m_), cn = nrm2(c_s, n_);
    return (hn > 1e-10 && cn > 1e-10) ? cn / hn : 1.0;
  }
  void run_until_halt();
  void setup_fp32();
  // FP32 mode: fix FP64 anchors at the current iterates (mask: instances, NULL = all)
  void anchor(const int32_t* ix, const int32_t* iy, const uint8_t* mask);
  // FP32 mode: fold the deltas back into the FP64 iterates
  void materialize(const int32_t* ix, const int32_t* iy, const uint8_t* mask);
  void main_loop();
  double power_method(bool* converged);
  void resolving();
  void omega_update(double* xds, double* yds, bool clamp);
  void log_progress();
};

// ---------------------------------------------------------------------------
int Solver::validate() {
  if (P.n < 0 || P.m < 0 || P.nb < 0 || P.nb > P.n || P.nnz < 0) return PDCS_ERR_INVALID;
  if ((P.m > 0 && (!P.G_rowptr || !P.h)) || (P.n > 0 && !P.c) || (P.nnz > 0 && (!P.G_colind || !P.G_val)))
    return PDCS_ERR_INVALID;
  if (P.nb > 0 && (!P.bl || !P.bu)) return PDCS_ERR_INVALID;
  if (P.nnz > INT32_MAX || P.n > INT32_MAX || P.m > INT32_MAX) return PDCS_ERR_INVALID;
  int64_t msum = P.mGzero + P.mGnonnegative + 3 * (P.expG + P.dual_expG);
  for (int64_t i = 0; i < P.n_socG; ++i) msum += P.socG[i];
  for (int64_t i = 0; i < P.n_rsocG; ++i) msum += P.rsocG[i];
  if (msum != P.m) return PDCS_ERR_M_MISMATCH;
  for (int64_t i = 0; i < P.n_socG; ++i) if (P.socG[i] < 2) return PDCS_ERR_SOC_DIM;
  for (int64_t i = 0; i < P.n_soc_x; ++i) if (P.soc_x[i] < 2) return PDCS_ERR_SOC_DIM;
  for (int64_t i = 0; i < P.n_rsocG; ++i) if (P.rsocG[i] < 3) return PDCS_ERR_RSOC_DIM;
  for (int64_t i = 0; i < P.n_rsoc_x; ++i) if (P.rsoc_x[i] < 3) return PDCS_ERR_RSOC_DIM;
  int64_t nsum = P.nb + 3 * (P.exp_x + P.dual_exp_x);
  for (int64_t i = 0; i < P.n_soc_x; ++i) nsum += P.soc_x[i];
  for (int64_t i = 0; i < P.n_rsoc_x; ++i) nsum += P.rsoc_x[i];
  if (nsum > P.n) return PDCS_ERR_N_MISMATCH;
  if (O.use_preconditioner == 0 || O.use_adaptive_restart == 0 || O.use_adaptive_step_size_weight == 0 ||
      O.use_aggressive == 0 || O.use_accelerated != 0 || (O.precision != 0 && O.precision != 1))
    return PDCS_ERR_UNSUPPORTED;  // only the reference GPU module's live main loop (rpdhg_alg_gpu_gen.jl:1886-1927)
  return PDCS_OK;
}

// Rows binned by length for a schedule of lane_nnz nonzeros per lane: bin b < 6
// takes rows of at most lane_nnz * 2^b nonzeros (g = 2^b lanes each), bin 6 the
// longer rows (a CTA each), bin 7 the chunks of rows over kSplitMin nonzeros
// (one instance only: the batched solver's masked SpMV keeps them in bin 6).
// Counting sort: rows keep their order inside a bin.
void Solver::build_bins(const std::vector<int32_t>& rp, int64_t rows, int64_t cols, const int32_t* d_rp,
                        const int32_t* d_ci, const double* d_v, CsrDev& D, const int32_t* row_inst, int lane_nnz) {
  D.m = rows;
  D.n = cols;
  D.nnz = rp[rows];
  D.rp = d_rp;
  D.ci = d_ci;
  D.v = d_v;
  D.dbin = nullptr;
  D.lane_nnz = lane_nnz;
  const bool split = row_inst == nullptr;
  auto bin_of = [&](int64_t i) {
    const int64_t L = rp[i + 1] - rp[i];
    if (split && L > kSplitMin) return kSplitBin;
    if (L > 32LL * lane_nnz) return kRowBin;
    int b = 0;
    while (b < kRowBin - 1 && ((int64_t)lane_nnz << b) < L) ++b;
    return b;
  };
  auto chunks = [&](int64_t i) { return (rp[i + 1] - rp[i] + kSplitChunk - 1) / kSplitChunk; };
  int64_t cnt[kBins] = {};
  for (int64_t i = 0; i < rows; ++i) {
    const int b = bin_of(i);
    cnt[b] += b == kSplitBin ? chunks(i) : 1;
  }
  int64_t off = 0;
  int32_t cta = 0;
  int64_t pos[kBins];
  for (int b = 0; b < kBins; ++b) {
    D.bin_off[b] = off;
    D.cta0[b] = cta;
    pos[b] = off;
    const int64_t R = cnt[b];
    off += R;
    if (R == 0) continue;
    if (b < kRowBin) {
      int64_t rows_per_cta = kThreads >> b;
      cta += (int32_t)std::min<int64_t>((R + rows_per_cta - 1) / rows_per_cta, 148 * 16);
    } else if (b == kRowBin) {
      cta += (int32_t)std::min<int64_t>(R, 148 * 8);
    } else {  // a CTA per chunk: resident CTAs in different phases keep the loads streaming
      cta += (int32_t)std::min<int64_t>(R, 1 << 24);
    }
  }
  D.bin_off[kBins] = off;
  D.cta0[kBins] = std::max(cta, 1);
  std::vector<int4> desc(off);
  int32_t slot = 0;
  for (int64_t i = 0; i < rows; ++i) {
    const int b = bin_of(i);
    if (b == kSplitBin) {
      for (int64_t k = rp[i]; k < rp[i + 1]; k += kSplitChunk)
        desc[pos[b]++] = make_int4((int32_t)i, (int32_t)k, (int32_t)std::min<int64_t>(k + kSplitChunk, rp[i + 1]), slot++);
    } else {
      desc[pos[b]++] = make_int4((int32_t)i, rp[i], rp[i + 1], row_inst ? row_inst[i] : 0);
    }
  }
  D.spart = nullptr;
  D.scnt = nullptr;
  if (slot > 0) {  // one workspace per matrix, shared by its schedules (same chunks)
    auto it = split_ws_.find(d_rp);
    if (it == split_ws_.end()) {
      double* p = A.alloc<double>(2 * (size_t)slot);
      unsigned* c = A.alloc<unsigned>(slot);
      PDCS_CUDA(cudaMemsetAsync(c, 0, sizeof(unsigned) * slot, s_));
      it = split_ws_.emplace(d_rp, std::make_pair(p, c)).first;
    }
    D.spart = it->second.first;
    D.scnt = it->second.second;
  }
  int4* d_desc = A.alloc<int4>(std::max<size_t>(desc.size(), 1));
  if (!desc.empty())
    PDCS_CUDA(cudaMemcpyAsync(d_desc, desc.data(), desc.size() * sizeof(int4), cudaMemcpyHostToDevice, s_));
  PDCS_CUDA(cudaStreamSynchronize(s_));  // the host vector is released on return
  D.rows = d_desc;
}

// matrices with fewer nonzeros keep the default schedule: timing four candidates
// costs more than a small solve can gain from the choice
constexpr int64_t kTuneMinNnz = 1 << 20;

// FP32 view of a CSR with the same structure and schedule
static CsrT<float> narrow_csr(const CsrDev& D, const float* v) {
  CsrT<float> F;
  F.m = D.m;
  F.n = D.n;
  F.nnz = D.nnz;
  F.rp = D.rp;
  F.ci = D.ci;
  F.v = v;
  F.rows = D.rows;
  F.dbin = D.dbin;
  F.lane_nnz = D.lane_nnz;
  F.spart = D.spart;
  F.scnt = D.scnt;
  for (int b = 0; b <= kBins; ++b) {
    F.bin_off[b] = D.bin_off[b];
    F.cta0[b] = D.cta0[b];
  }
  return F;
}

// SpMV schedule autotuner: time each nonzeros-per-lane target on this matrix
// (CUDA events, best of 3 after a warm-up) and keep the fastest, leaving the
// default (4) only for a gain of 3% or more; a fixed target (spmv_lane_nnz > 0)
// skips the search.  The choice is remembered per device and row structure
// for the life of the process, so repeated solves of a matrix use the same
// schedule (and give bit-identical results).  With v32 (FP32-bulk mode) the
// candidates are timed on the FP32 values, the precision of the iteration.
// Returns the target used.
int Solver::tune_bins(const std::vector<int32_t>& rp, int64_t rows, int64_t cols, const int32_t* d_rp,
                      const int32_t* d_ci, const double* d_v, CsrDev& D, const int32_t* row_inst, const double* xin,
                      double* yout, const float* v32) {
  if (O.spmv_lane_nnz > 0 || rp[rows] < kTuneMinNnz) {  // fixed, or too small for the search to pay off
    const int lane = O.spmv_lane_nnz > 0 ? O.spmv_lane_nnz : 4;
    build_bins(rp, rows, cols, d_rp, d_ci, d_v, D, row_inst, lane);
    return lane;
  }
  static std::mutex mu;
  static std::map<std::array<uint64_t, 5>, int> chosen;
  int dev = 0;
  PDCS_CUDA(cudaGetDevice(&dev));
  uint64_t h = 1469598103934665603ull;
  for (int64_t i = 0; i <= rows; ++i) {
    h ^= (uint64_t)(uint32_t)rp[i];
    h *= 1099511628211ull;
  }
  const std::array<uint64_t, 5> key{(uint64_t)dev, (uint64_t)rows, (uint64_t)cols, h, v32 ? 1ull : 0ull};
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = chosen.find(key);
    if (it != chosen.end()) {
      build_bins(rp, rows, cols, d_rp, d_ci, d_v, D, row_inst, it->second);
      return it->second;
    }
  }
  cudaEvent_t e0, e1;
  PDCS_CUDA(cudaEventCreate(&e0));
  PDCS_CUDA(cudaEventCreate(&e1));
  int best = 4;
  float best_ms = 1e30f;
  CsrDev best_D{};
  float *x32 = nullptr, *y32 = nullptr;
  if (v32) {
    x32 = A.alloc<float>(cols);
    y32 = A.alloc<float>(rows);
    PDCS_CUDA(cudaMemsetAsync(x32, 0, sizeof(float) * std::max<int64_t>(cols, 1), s_));
  }
  for (int lane : {4, 2, 8, 16}) {  // the default first: others must beat it by 3%
    CsrDev C;
    build_bins(rp, rows, cols, d_rp, d_ci, d_v, C, row_inst, lane);
    const CsrT<float> C32 = narrow_csr(C, v32);
    auto run = [&]() {
      if (v32)
        launch_spmv<1>(C32, x32, nullptr, y32, nullptr, nullptr, s_);
      else
        spmv(C, xin, yout);
    };
    run();
    float t = 1e30f;
    for (int r = 0; r < 3; ++r) {
      PDCS_CUDA(cudaEventRecord(e0, s_));
      run();
      PDCS_CUDA(cudaEventRecord(e1, s_));
      PDCS_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      PDCS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      t = std::min(t, ms);
    }
    if (!v32) kernels_ -= 4;
    if (lane != 4) t *= 1.03f;
    if (t < best_ms) {
      if (best_D.rows) A.drop(best_D.rows);
      best_ms = t;
      best = lane;
      best_D = C;
    } else {
      A.drop(C.rows);
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (x32) {
    A.drop(x32);
    A.drop(y32);
  }
  D = best_D;
  std::lock_guard<std::mutex> lock(mu);
  chosen.emplace(key, best);
  return best;
}

void Solver::size_table(ConeTable& T) {
  T.elem_total = 0;
  for (int s = 0; s < T.nseg; ++s) T.elem_total += T.seg_len[s];
  auto cap = [](int64_t v) { return (int32_t)std::min<int64_t>(v, 148 * 8); };
  T.ctaA = T.elem_total > 0 ? cap((T.elem_total + kThreads - 1) / kThreads) : 0;
  const int64_t tasks = T.task0[kCls];
  T.ctaB = tasks > 0 ? cap((tasks + kWarps - 1) / kWarps) : 0;
  int64_t ne = T.exp_count + T.dexp_count;
  T.ctaC = ne > 0 ? cap((ne + kThreads - 1) / kThreads) : 0;
  T.ctaD = 0;
  if (T.nhuge > 0) {
    int64_t dmin = T.huge_len[0];
    for (int h = 1; h < T.nhuge; ++h) dmin = std::min(dmin, T.huge_len[h]);
    // about 2048 elements per CTA, at most two CTAs per SM (every CTA of part D resident),
    // at least 2 elements per CTA (elements 0 and 1 of a block in CTA 0)
    T.ctaD = (int32_t)std::max<int64_t>(1, std::min<int64_t>({(dmin + 2047) / 2048, dmin / 2, (int64_t)kHugeMaxCtas}));
    if (!huge_bar_) {
      huge_bar_ = A.alloc<unsigned>(4);
      huge_err_ = A.alloc<int32_t>(4);
      huge_red_ = A.alloc<double>(2 * 4 * kHugeMaxCtas);
      PDCS_CUDA(cudaMemsetAsync(huge_bar_, 0, 4 * sizeof(unsigned), s_));
      PDCS_CUDA(cudaMemsetAsync(huge_err_, 0, 4 * sizeof(int32_t), s_));
    }
    T.huge_bar = huge_bar_;
    T.huge_err = huge_err_;
    T.huge_red = huge_red_;
    int64_t tot = 0;
    for (int h = 0; h < T.nhuge; ++h) {
      T.huge_soff[h] = tot;
      tot += T.huge_len[h];
    }
    T.huge_scr = A.alloc<double2>(tot);
  }
  if (table_grid(T) == 0) T.ctaA = 1;  // at least one CTA writes the partials
}

void Solver::build_tables(const std::vector<int64_t>& soc_x, const std::vector<int64_t>& rsoc_x,
                          const std::vector<int64_t>& socG, const std::vector<int64_t>& rsocG) {
  // warp-cone lists (shared by the iteration and KKT tables of each vector)
  // warp-cone lists and their size-class schedule (lane groups of cls_lanes(c) lanes)
  auto upload_wc = [&](const std::vector<int64_t>& soc, const std::vector<int64_t>& rsoc, int64_t start0,
                       ConeTable& T) {
    std::vector<int64_t> stv;
    std::vector<int32_t> lv;
    std::vector<int8_t> kv;
    int64_t s = start0;
    for (int64_t d : soc) { stv.push_back(s); lv.push_back((int32_t)d); kv.push_back(PK_SOC); s += d; }
    for (int64_t d : rsoc) { stv.push_back(s); lv.push_back((int32_t)d); kv.push_back(PK_RSOC); s += d; }
    std::vector<std::vector<int64_t>> cls(kCls);
    T.nhuge = 0;
    for (size_t k = 0; k < lv.size(); ++k) {
      // part D (the launch's first CTAs together) in the single solver; the batched
      // solver's masked updates keep every block on a warp (part D ignores the mask)
      if (lv[k] >= kHugeBlock && T.nhuge < kMaxHuge && inst_of_y_ == nullptr) {
        T.huge_start[T.nhuge] = stv[k];
        T.huge_len[T.nhuge] = lv[k];
        T.huge_rsoc[T.nhuge] = kv[k] == PK_RSOC ? 1 : 0;
        T.huge_wc[T.nhuge] = (int64_t)k;
        T.nhuge++;
        continue;
      }
      int c = 0;
      while (c < kCls - 1 && lv[k] > (2 << c)) ++c;
      cls[c].push_back((int64_t)k);
    }
    std::vector<int64_t> sched;
    int64_t task = 0;
    for (int c = 0; c < kCls; ++c) {
      T.cls_off[c] = (int64_t)sched.size();
      T.task0[c] = task;
      sched.insert(sched.end(), cls[c].begin(), cls[c].end());
      const int64_t per = (c < kCls - 1) ? 32 / cls_lanes(c) : 1;
      task += ((int64_t)cls[c].size() + per - 1) / per;
    }
    T.cls_off[kCls] = (int64_t)sched.size();
    T.task0[kCls] = task;
    int64_t* d_start = A.alloc<int64_t>(stv.size());
    int32_t* d_len = A.alloc<int32_t>(lv.size());
    int8_t* d_kind = A.alloc<int8_t>(kv.size());
    int64_t* d_sched = A.alloc<int64_t>(std::max<size_t>(sched.size(), 1));
    if (!stv.empty()) {
      PDCS_CUDA(cudaMemcpyAsync(d_start, stv.data(), stv.size() * sizeof(int64_t), cudaMemcpyHostToDevice, s_));
      PDCS_CUDA(cudaMemcpyAsync(d_len, lv.data(), lv.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s_));
      PDCS_CUDA(cudaMemcpyAsync(d_kind, kv.data(), kv.size() * sizeof(int8_t), cudaMemcpyHostToDevice, s_));
      PDCS_CUDA(cudaMemcpyAsync(d_sched, sched.data(), sched.size() * sizeof(int64_t), cudaMemcpyHostToDevice, s_));
      PDCS_CUDA(cudaStreamSynchronize(s_));
    }
    T.nwc = (int64_t)stv.size();
    T.wc_start = d_start;
    T.wc_len = d_len;
    T.wc_kind = d_kind;
    T.sched = d_sched;
    return s;
  };
  ConeTable base_x{};
  ConeTable base_y{};
  int64_t xe = upload_wc(soc_x, rsoc_x, nb_, base_x);
  int64_t ye = upload_wc(socG, rsocG, P.mGzero + P.mGnonnegative, base_y);
  base_x.len = n_;
  base_x.exp_base = xe;
  base_x.exp_count = P.exp_x;
  base_x.dexp_base = xe + 3 * P.exp_x;
  base_x.dexp_count = P.dual_exp_x;
  if (nb_ > 0) {
    base_x.nseg = 1;
    base_x.seg_start[0] = 0;
    base_x.seg_len[0] = nb_;
    base_x.seg_kind[0] = PK_BOX;
  }
  XI = base_x;
  XI.lo = bl_s;
  XI.hi = bu_s;
  XI.exp_kind = PK_EXP;    // code 27
  XI.dexp_kind = PK_DEXP;  // code 29
  XI.S = Dr;
  SLK = base_x;
  SLK.lo = lam_l;
  SLK.hi = lam_u;
  SLK.exp_kind = PK_DEXP;  // code 28
  SLK.dexp_kind = PK_EXP;  // code 26
  SLK.S = nullptr;
  base_y.len = m_;
  base_y.exp_base = ye;
  base_y.exp_count = P.expG;
  base_y.dexp_base = ye + 3 * P.expG;
  base_y.dexp_count = P.dual_expG;
  int ns = 0;
  if (P.mGzero > 0) {
    base_y.seg_start[ns] = 0;
    base_y.seg_len[ns] = P.mGzero;
    ns++;
  }
  if (P.mGnonnegative > 0) {
    base_y.seg_start[ns] = P.mGzero;
    base_y.seg_len[ns] = P.mGnonnegative;
    base_y.seg_kind[ns] = PK_NONNEG;
    ns++;
  }
  base_y.nseg = ns;
  YI = base_y;
  CON = base_y;
  if (P.mGzero > 0) {
    YI.seg_kind[0] = PK_FREE;   // code 1
    CON.seg_kind[0] = PK_ZERO;  // code 2
  }
  YI.exp_kind = PK_DEXP;   // code 12: y in Dl o K_exp^*
  YI.dexp_kind = PK_EXP;   // code 15
  YI.S = Dl;
  CON.exp_kind = PK_EXP;   // code 13
  CON.dexp_kind = PK_DEXP; // code 16
  CON.S = nullptr;
  // per-cone warm starts of the exponential-cone root (NaN = none yet)
  int64_t nxe = P.exp_x + P.dual_exp_x, nye = P.expG + P.dual_expG;
  XI.rho_ws = A.alloc<double>(nxe);
  YI.rho_ws = A.alloc<double>(nye);
  PDCS_CUDA(cudaMemsetAsync(XI.rho_ws, 0xff, sizeof(double) * std::max<int64_t>(nxe, 1), s_));
  PDCS_CUDA(cudaMemsetAsync(YI.rho_ws, 0xff, sizeof(double) * std::max<int64_t>(nye, 1), s_));
  // per-block warm starts of the weighted-SOC root (the unscaled tables use the closed form)
  XI.soc_ws = A.alloc<double>(std::max<int64_t>(XI.nwc, 1));
  YI.soc_ws = A.alloc<double>(std::max<int64_t>(YI.nwc, 1));
  PDCS_CUDA(cudaMemsetAsync(XI.soc_ws, 0xff, sizeof(double) * std::max<int64_t>(XI.nwc, 1), s_));
  PDCS_CUDA(cudaMemsetAsync(YI.soc_ws, 0xff, sizeof(double) * std::max<int64_t>(YI.nwc, 1), s_));
  size_table(XI);
  size_table(SLK);
  size_table(YI);
  size_table(CON);
}

void Solver::setup() {
  n_ = P.n;
  m_ = P.m;
  nb_ = P.nb;
  nnz_ = P.nnz;
  if (O.stream) {
    s_ = static_cast<cudaStream_t>(O.stream);
  } else {
    PDCS_CUDA(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking));
    own_stream_ = true;
  }
  A.bind(s_);
  phase_t_ = 0.0;
  phase("start");
  PDCS_CUDA(cudaMallocHost(&host_state_, sizeof(PdhgState)));
  PDCS_CUDA(cudaMallocHost(&host_red_, 64 * sizeof(double)));
  part_r = A.alloc<double>((size_t)148 * 8 * 8);
  red_out = A.alloc<double>(64);
  // ---- raw problem data on the device (copied: the caller's buffers are never modified) ----
  int32_t* g_rp = A.alloc<int32_t>(m_ + 1);
  int32_t* g_ci = A.alloc<int32_t>(nnz_);
  double* g_v = A.alloc<double>(nnz_);
  c_raw = A.alloc<double>(n_);
  h_raw = A.alloc<double>(m_);
  double* bl_raw = A.alloc<double>(nb_);
  double* bu_raw = A.alloc<double>(nb_);
  bl_raw_ = bl_raw;
  bu_raw_ = bu_raw;
  const cudaMemcpyKind kind = P.on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  auto put = [&](void* dst, const void* src, size_t bytes) {
    if (bytes) PDCS_CUDA(cudaMemcpyAsync(dst, src, bytes, kind, s_));
  };
  upload_matrix(g_rp, g_ci, g_v);
  put(c_raw, P.c, sizeof(double) * n_);
  put(h_raw, P.h, sizeof(double) * m_);
  put(bl_raw, P.bl, sizeof(double) * nb_);
  put(bu_raw, P.bu, sizeof(double) * nb_);
  phase("upload");
  // ---- input checks ----
  int32_t* d_err = A.alloc<int32_t>(1);
  PDCS_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int32_t), s_));
  check_inputs_kernel<<<grid_for(std::max(std::max(m_, nnz_), nb_)), kThreads, 0, s_>>>(m_, n_, nnz_, nb_, g_rp, g_ci,
                                                                                        bl_raw, bu_raw, d_err);
  int32_t* h_err = reinterpret_cast<int32_t*>(host_red_);
  PDCS_CUDA(cudaMemcpyAsync(h_err, d_err, sizeof(int32_t), cudaMemcpyDeviceToHost, s_));
  PDCS_CUDA(cudaStreamSynchronize(s_));
  if (*h_err & IE_BOUNDS) throw std::domain_error("bounds");
  if (*h_err) throw std::invalid_argument("csr");
  // raw norms (cal_constant, def_struct.jl:968-976)
  {
    DotSpec d{};
    d.a[0] = h_raw; d.kind[0] = DK_SUMABS;
    d.a[1] = h_raw; d.kind[1] = DK_MAXABS;
    d.count = 2; d.len = m_;
    double r[2];
    dots(d, r);
    hNrm1 = r[0];
    hNrmInf = r[1];
    DotSpec e{};
    e.a[0] = c_raw; e.kind[0] = DK_SUMABS;
    e.a[1] = c_raw; e.kind[1] = DK_MAXABS;
    e.count = 2; e.len = n_;
    dots(e, r);
    cNrm1 = r[0];
    cNrmInf = r[1];
  }
  phase("input checks, norms");
  // ---- G' structure: stable radix sort of the column keys keeps G's row order ----
  int32_t* row_of = A.alloc<int32_t>(nnz_);
  int32_t* t_rp = A.alloc<int32_t>(n_ + 1);
  int32_t* col_cnt = A.alloc<int32_t>(n_ + 1);
  int32_t* keys_sorted = A.alloc<int32_t>(nnz_);
  int32_t* perm_in = A.alloc<int32_t>(nnz_);
  int32_t* perm_t = A.alloc<int32_t>(nnz_);
  PDCS_CUDA(cudaMemsetAsync(col_cnt, 0, sizeof(int32_t) * (n_ + 1), s_));
  PDCS_CUDA(cudaMemsetAsync(perm_in, 0, sizeof(int32_t) * std::max<int64_t>(nnz_, 1), s_));
  row_start_kernel<<<grid_for(m_), kThreads, 0, s_>>>(m_, g_rp, perm_in);
  col_count_kernel<<<grid_for(nnz_), kThreads, 0, s_>>>(nnz_, g_ci, col_cnt);
  {
    size_t b1 = 0, b2 = 0, b3 = 0;
    int bits = 1;
    while ((int64_t(1) << bits) <= n_) ++bits;
    PDCS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, b1, col_cnt, t_rp, (int)(n_ + 1), s_));
    PDCS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b2, g_ci, keys_sorted, perm_in, perm_t, (int)nnz_, 0, bits,
                                              s_));
    PDCS_CUDA(cub::DeviceScan::InclusiveScan(nullptr, b3, perm_in, row_of, MaxI32{}, (int)nnz_, s_));
    void* tmp = A.alloc<char>(std::max(std::max(b1, b2), b3));
    if (nnz_ > 0) PDCS_CUDA(cub::DeviceScan::InclusiveScan(tmp, b3, perm_in, row_of, MaxI32{}, (int)nnz_, s_));
    iota_kernel<<<grid_for(nnz_), kThreads, 0, s_>>>(perm_in, nnz_);
    PDCS_CUDA(cub::DeviceScan::ExclusiveSum(tmp, b1, col_cnt, t_rp, (int)(n_ + 1), s_));
    if (nnz_ > 0)
      PDCS_CUDA(cub::DeviceRadixSort::SortPairs(tmp, b2, g_ci, keys_sorted, perm_in, perm_t, (int)nnz_, 0, bits, s_));
  }
  // both row-pointer arrays on the host (row bins, and the long rows of the statistics below)
  std::vector<int32_t> rp_h(m_ + 1), trp_h(n_ + 1);
  PDCS_CUDA(cudaMemcpyAsync(rp_h.data(), g_rp, sizeof(int32_t) * (m_ + 1), cudaMemcpyDeviceToHost, s_));
  PDCS_CUDA(cudaMemcpyAsync(trp_h.data(), t_rp, sizeof(int32_t) * (n_ + 1), cudaMemcpyDeviceToHost, s_));
  PDCS_CUDA(cudaStreamSynchronize(s_));
  // rows (of G and of G') over kStatLong nonzeros: a CTA each in the row statistics
  constexpr int64_t kStatLong = 4096;
  auto long_rows = [&](const std::vector<int32_t>& rp, int64_t rows, int64_t& count) -> int32_t* {
    std::vector<int32_t> l;
    for (int64_t i = 0; i < rows; ++i)
      if (rp[i + 1] - rp[i] > kStatLong) l.push_back((int32_t)i);
    count = (int64_t)l.size();
    if (l.empty()) return nullptr;
    int32_t* d = A.alloc<int32_t>(l.size());
    PDCS_CUDA(cudaMemcpyAsync(d, l.data(), sizeof(int32_t) * l.size(), cudaMemcpyHostToDevice, s_));
    PDCS_CUDA(cudaStreamSynchronize(s_));
    return d;
  };
  int64_t nlong_g = 0, nlong_t = 0;
  int32_t* long_g = long_rows(rp_h, m_, nlong_g);
  int32_t* long_t = long_rows(trp_h, n_, nlong_t);
  phase("transpose");
  // ---- Ruiz (10) + Pock-Chambolle (alpha = 1) equilibration on the device ----
  c_s = A.alloc<double>(n_);
  Dr = A.alloc<double>(n_);
  h_s = A.alloc<double>(m_);
  Dl = A.alloc<double>(m_);
  bl_s = A.alloc<double>(nb_);
  bu_s = A.alloc<double>(nb_);
  copy(c_s, c_raw, n_);
  copy(h_s, h_raw, m_);
  copy(bl_s, bl_raw, nb_);
  copy(bu_s, bu_raw, nb_);
  double* g_v_raw = nullptr;
  if (O.differentiable) {  // the adjoint differentiates the unscaled problem
    g_v_raw = A.alloc<double>(nnz_);
    copy(g_v_raw, g_v, nnz_);
  }
  fill_kernel<<<grid_for(n_), kThreads, 0, s_>>>(Dr, 1.0, n_);
  fill_kernel<<<grid_for(m_), kThreads, 0, s_>>>(Dl, 1.0, m_);
  double* var = A.alloc<double>(n_);
  double* con = A.alloc<double>(m_);
  auto stat = [&](auto sum_tag, int64_t rows, const int32_t* rp, const int32_t* perm, double* out,
                  const int32_t* list, int64_t nlist) {
    constexpr bool SUM = decltype(sum_tag)::value;
    row_absstat_kernel<SUM><<<warp_grid(rows), kThreads, 0, s_>>>(rows, rp, g_v, perm, out, list ? kStatLong : -1);
    if (list)
      row_absstat_long_kernel<SUM><<<(int)std::min<int64_t>(nlist, 148 * 8), kThreads, 0, s_>>>(nlist, list, rp, g_v,
                                                                                                perm, out);
  };
  auto pass = [&](bool sum) {
    if (sum) {
      stat(std::true_type{}, m_, g_rp, nullptr, con, long_g, nlong_g);
      stat(std::true_type{}, n_, t_rp, perm_t, var, long_t, nlong_t);
    } else {
      stat(std::false_type{}, m_, g_rp, nullptr, con, long_g, nlong_g);
      stat(std::false_type{}, n_, t_rp, perm_t, var, long_t, nlong_t);
    }
    sqrt_or_one_kernel<<<grid_for(m_), kThreads, 0, s_>>>(con, m_);
    sqrt_or_one_kernel<<<grid_for(n_), kThreads, 0, s_>>>(var, n_);
    scale_matrix_kernel<<<grid_for(nnz_), kThreads, 0, s_>>>(nnz_, row_of, g_ci, g_v, con, var);
    scale_vectors_kernel<<<grid_for(std::max(n_, m_)), kThreads, 0, s_>>>(n_, nb_, m_, var, con, c_s, Dr, bl_s, bu_s,
                                                                        h_s, Dl);
  };
  int method = O.rescaling_method;
  if (method == 1 || method == 3)
    for (int it = 0; it < 10; ++it) pass(false);
  if (method == 2 || method == 3) pass(true);
  int32_t* t_ci = A.alloc<int32_t>(nnz_);
  double* t_v = A.alloc<double>(nnz_);
  gather_transpose_kernel<<<grid_for(nnz_), kThreads, 0, s_>>>(nnz_, perm_t, row_of, g_v, t_ci, t_v);
  {
    DotSpec d{};
    d.a[0] = g_v; d.kind[0] = DK_MAXABS;
    d.count = 1; d.len = nnz_;
    dots(d, &ginf_);
  }
  lam_l = A.alloc<double>(nb_); lam_u = A.alloc<double>(nb_);
  bl_fin = A.alloc<double>(nb_); bu_fin = A.alloc<double>(nb_);
  if (nb_ > 0)
    box_aux_kernel<<<grid_for(nb_), kThreads, 0, s_>>>(nb_, bl_raw, bu_raw, bl_fin, bu_fin, lam_l, lam_u);
  phase("equilibration");
  // ---- iterates and work vectors ----
  auto vecn = [&]() { return A.alloc<double>(n_); };
  auto vecm = [&]() { return A.alloc<double>(m_); };
  x = vecn(); xl = vecn(); xm = vecn(); aty = vecn(); x0 = vecn(); x0l = vecn(); xbest = vecn();
  y = vecm(); yl = vecm(); ym = vecm(); gx = vecm(); gxl = vecm(); y0 = vecm(); y0l = vecm(); ybest = vecm();
  for (int k = 0; k < 6; ++k) { tn[k] = vecn(); tm[k] = vecm(); }
  xds_ = vecn();
  yds_ = vecm();
  // initial point: zeros, or the warm start scaled into the preconditioned space
  if (O.warm_start && O.primal_sol && O.dual_sol) {
    PDCS_CUDA(cudaMemcpyAsync(x, O.primal_sol, sizeof(double) * n_, cudaMemcpyHostToDevice, s_));
    PDCS_CUDA(cudaMemcpyAsync(y, O.dual_sol, sizeof(double) * m_, cudaMemcpyHostToDevice, s_));
    mul_kernel<<<grid_for(n_), kThreads, 0, s_>>>(x, Dr, n_);
    mul_kernel<<<grid_for(m_), kThreads, 0, s_>>>(y, Dl, m_);
  } else {
    if (n_) PDCS_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n_, s_));
    if (m_) PDCS_CUDA(cudaMemsetAsync(y, 0, sizeof(double) * m_, s_));
  }
  copy(xl, x, n_); copy(xm, x, n_); copy(xbest, x, n_);
  copy(yl, y, m_); copy(ym, y, m_); copy(ybest, y, m_);
  phase("row bins, work vectors");
  // ---- SpMV schedules: autotuned per matrix unless fixed by the options ----
  if (O.precision == 1) {  // the FP32 iteration sets the schedule
    gv32_ = A.alloc<float>(nnz_);
    tv32_ = A.alloc<float>(nnz_);
    to_float_kernel<<<grid_for(nnz_), kThreads, 0, s_>>>(gv32_, g_v, nnz_);
    to_float_kernel<<<grid_for(nnz_), kThreads, 0, s_>>>(tv32_, t_v, nnz_);
  }
  lane_G_ = tune_bins(rp_h, m_, n_, g_rp, g_ci, g_v, G_, inst_of_y_, x, tm[0], gv32_);
  lane_Gt_ = tune_bins(trp_h, n_, m_, t_rp, t_ci, t_v, Gt_, inst_of_x_, y, tn[0], tv32_);
  if (O.differentiable) {
    double* t_v_raw = A.alloc<double>(nnz_);
    gather_kernel<<<grid_for(nnz_), kThreads, 0, s_>>>(t_v_raw, g_v_raw, perm_t, nnz_);
    Graw_ = G_;
    Graw_.v = g_v_raw;
    Gtraw_ = Gt_;
    Gtraw_.v = t_v_raw;
  }
  // cone tables
  std::vector<int64_t> soc_x(P.soc_x, P.soc_x + P.n_soc_x), rsoc_x(P.rsoc_x, P.rsoc_x + P.n_rsoc_x);
  std::vector<int64_t> socG(P.socG, P.socG + P.n_socG), rsocG(P.rsocG, P.rsocG + P.n_rsocG);
  phase("SpMV schedules");
  build_tables(soc_x, rsoc_x, socG, rsocG);
  int maxgrid = std::max({table_grid(XI), table_grid(YI), table_grid(SLK), table_grid(CON), 148 * 8});
  part_x = A.alloc<double>((size_t)maxgrid * 8);
  part_y = A.alloc<double>((size_t)maxgrid * 8);
  part_r = A.alloc<double>((size_t)maxgrid * 8);
  part_a = A.alloc<double>((size_t)maxgrid * 8);
  part_b = A.alloc<double>((size_t)maxgrid * 8);
  st_dev = A.alloc<PdhgState>(1);
  PDCS_CUDA(cudaMemsetAsync(st_dev, 0, sizeof(PdhgState), s_));
  grid_reflect_ = grid_for(std::max(n_, m_));
  attempts_per_graph_ = O.attempts_per_graph > 0 ? O.attempts_per_graph : 32;
  phase("cone tables");
  if (O.precision == 1) setup_fp32();
  phase("FP32 copies");
  PDCS_CUDA(cudaStreamSynchronize(s_));
}

void Solver::setup_fp32() {
  fp32_ = true;
  if (!gv32_) {
    gv32_ = A.alloc<float>(nnz_);
    tv32_ = A.alloc<float>(nnz_);
    to_float_kernel<<<grid_for(nnz_), kThreads, 0, s_>>>(gv32_, G_.v, nnz_);
    to_float_kernel<<<grid_for(nnz_), kThreads, 0, s_>>>(tv32_, Gt_.v, nnz_);
  }
  G32_ = narrow_csr(G_, gv32_);
  Gt32_ = narrow_csr(Gt_, tv32_);
  dxp32_ = A.alloc<float2>(n_);
  aty32_ = A.alloc<float>(n_);
  dy32_ = A.alloc<float>(m_);
  dyl32_ = A.alloc<float>(m_);
  gx32_ = A.alloc<float>(m_);
  gxl32_ = A.alloc<float>(m_);
  xa_ = A.alloc<double>(n_);
  qa_ = A.alloc<double>(n_);
  dxm_ = A.alloc<double>(n_);
  ya_ = A.alloc<double>(m_);
  ra_ = A.alloc<double>(m_);
  dym_ = A.alloc<double>(m_);
}

void Solver::anchor(const int32_t* ix, const int32_t* iy, const uint8_t* mask) {
  anchor_kernel<<<grid_for(n_), kThreads, 0, s_>>>(x, xl, xm, xa_, &dxp32_->x, &dxp32_->y, 2, dxm_, ix, mask, n_);
  anchor_kernel<<<grid_for(m_), kThreads, 0, s_>>>(y, yl, ym, ya_, dy32_, dyl32_, 1, dym_, iy, mask, m_);
  if (mask) {
    spmv_masked(Gt_, ya_, qa_, mask);
    spmv_masked(G_, xa_, ra_, mask);
  } else {
    spmv(Gt_, ya_, qa_);
    spmv(G_, xa_, ra_);
  }
  masked_sub_kernel<<<grid_for(n_), kThreads, 0, s_>>>(qa_, qa_, c_s, ix, mask, n_);
  masked_sub_kernel<<<grid_for(m_), kThreads, 0, s_>>>(ra_, ra_, h_s, iy, mask, m_);
  kernels_ += 4;
}

void Solver::materialize(const int32_t* ix, const int32_t* iy, const uint8_t* mask) {
  materialize_kernel<<<grid_for(n_), kThreads, 0, s_>>>(x, xl, xm, xa_, &dxp32_->x, &dxp32_->y, 2, dxm_, ix, mask,
                                                         n_);
  materialize_kernel<<<grid_for(m_), kThreads, 0, s_>>>(y, yl, ym, ya_, dy32_, dyl32_, 1, dym_, iy, mask, m_);
  kernels_ += 2;
}

void Solver::capture_graph() {
  PDCS_CUDA(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal));
  const int32_t* act = &st_dev->active;
  for (int a = 0; a < attempts_per_graph_ && fp32_; ++a) {
    launch_spmv<1, false, float>(Gt32_, dyl32_, nullptr, aty32_, nullptr, act, s_, &st_dev->do_reflect);
    OpPrimalStep32 op1{xa_, dxp32_, qa_, aty32_, x, st_dev, 0.0};
    launch_update_project(op1, XI, part_x, act, s_);
    launch_spmv<kPair, false, float>(G32_, &dxp32_->x, nullptr, gx32_, gxl32_, act, s_);
    OpDualStep32 op2{ya_, dyl32_, ra_, gx32_, gxl32_, dy32_, y, st_dev, 0.0, part_x, table_grid(XI)};
    launch_update_project(op2, YI, part_y, act, s_);
    reflect32_kernel<<<grid_reflect_, kThreads, 0, s_>>>(st_dev, dxp32_, dxm_, n_, dy32_, dyl32_, dym_, m_);
  }
  for (int a = 0; a < attempts_per_graph_ && !fp32_; ++a) {
    launch_spmv<1>(Gt_, yl, nullptr, aty, nullptr, act, s_, &st_dev->do_reflect);
    OpPrimalStep op1{xl, aty, c_s, x, st_dev, 0.0};
    launch_update_project(op1, XI, part_x, act, s_);
    launch_spmv<2>(G_, x, xl, gx, gxl, act, s_);
    // the dual step's last CTA runs the attempt's control step
    OpDualStep op2{yl, gx, gxl, h_s, y, st_dev, 0.0, part_x, table_grid(XI)};
    launch_update_project(op2, YI, part_y, act, s_);
    reflect_kernel<<<grid_reflect_, kThreads, 0, s_>>>(st_dev, x, xl, xm, n_, y, yl, ym, m_);
  }
  PDCS_CUDA(cudaStreamEndCapture(s_, &graph_));
  PDCS_CUDA(cudaGraphInstantiate(&graph_exec_, graph_, 0));
}

// converge_info_calculation_diagonal! (rpdhg_alg_gpu_gen_scaling.jl:126-183), on
// the scaled iterates: G_raw x_raw = Dl o (G~ x~),  G_raw' y_raw = Dr o (G~' y~).
void Solver::converge_info(const double* xs, const double* ys, Converge& C, double* gxs, double* atys) {
  spmv(G_, xs, gxs);
  spmv(Gt_, ys, atys);
  OpResidual opp{gxs, Dl, 1.0, nullptr, 0.0, h_raw, tm[5], bl_fin, bu_fin, 0};
  finalize_async(part_a, launch_project(opp, CON, part_a), 7, 0b0010110u, 0);
  OpResidual opd{atys, Dr, -1.0, c_raw, 1.0, nullptr, tn[5], bl_fin, bu_fin, nb_};
  finalize_async(part_b, launch_project(opd, SLK, part_b), 7, 0b0010110u, 7);
  DotSpec d1{};
  d1.a[0] = c_raw; d1.b[0] = xs; d1.sa[0] = Dr; d1.kind[0] = DK_DOT;  // c_raw' (x~ / Dr)
  d1.count = 1; d1.len = n_;
  dots_async(d1, part_r, 14);
  DotSpec d2{};
  d2.a[0] = h_raw; d2.b[0] = ys; d2.sa[0] = Dl; d2.kind[0] = DK_DOT;  // h_raw' (y~ / Dl)
  d2.count = 1; d2.len = m_;
  dots_async(d2, part_x, 15);
  const double* r = fetch(16);
  const double *rp = r, *rd = r + 7;
  double pobj = r[14], hy = r[15];
  double dobj = hy + rd[6];
  C.pobj = pobj;
  C.dobj = dobj;
  C.abs_gap = std::fabs(pobj - dobj);
  C.rel_gap = C.abs_gap / (1.0 + std::max(std::fabs(pobj), std::fabs(dobj)));
  double l2p = std::sqrt(rp[0]), linfp = rp[1], axinf = rp[4], axnrm1 = rp[5];
  double l2d = std::sqrt(rd[0]), linfd = rd[1], sinf = rd[2], snrm1 = rd[3], atyinf = rd[4], atynrm1 = rd[5];
  C.l2_abs_p = l2p;
  C.linf_abs_p = linfp;
  C.l2_abs_d = l2d;
  C.linf_abs_d = linfd;
  C.l2_rel_p = l2p / (1.0 + std::max(snrm1, std::max(hNrm1, axnrm1)));
  C.linf_rel_p = linfp / (1.0 + std::max(sinf, std::max(hNrmInf, axinf)));
  C.l2_rel_d = l2d / (1.0 + std::max(cNrm1, atynrm1));
  C.linf_rel_d = linfd / (1.0 + std::max(cNrmInf, atyinf));
}

// exit_condition_check_diagonal! (rpdhg_alg_gpu_gen_scaling.jl:309-352)
void Solver::exit_check() {
  Timer tm_(t_exit_);
  double *gxc = tm[0], *gxm = tm[1], *atc = tn[0], *atm = tn[1];
  converge_info(x, y, ci[0], gxc, atc);
  converge_info(xm, ym, ci[1], gxm, atm);
  check_count_++;
  // infeasibility information (rpdhg_alg_gpu_gen_scaling.jl:185-248).  For the
  // current iterate the rays are the iterates themselves, so the ray
  // infeasibilities equal the residuals just computed.
  auto push_trend = [&](Infea& I) {
    if (check_count_ % 4 == 1) {  // the reference pushes with probability 1/4
      I.ptrend.push_back(ci[0].pobj);
      I.dtrend.push_back(ci[0].dobj);
      if (I.ptrend.size() > 20) I.ptrend.erase(I.ptrend.begin());
      if (I.dtrend.size() > 20) I.dtrend.erase(I.dtrend.begin());
    }
  };
  // ray = current - average; G and G' of the difference by linearity
  double* dxs = tn[2];
  double* dys = tm[2];
  double* gd = tm[3];
  double* ad = tn[3];
  axpby(dxs, 1.0, x, -1.0, xm, n_);
  axpby(dys, 1.0, y, -1.0, ym, m_);
  axpby(gd, 1.0, gxc, -1.0, gxm, m_);
  axpby(ad, 1.0, atc, -1.0, atm, n_);
  DotSpec a{};  // n-length: |x/Dr|_inf, |dx/Dr|_inf, c'(dx/Dr)
  a.a[0] = x; a.sa[0] = Dr; a.kind[0] = DK_MAXABS;
  a.a[1] = dxs; a.sa[1] = Dr; a.kind[1] = DK_MAXABS;
  a.a[2] = c_raw; a.b[2] = dxs; a.sa[2] = Dr; a.kind[2] = DK_DOT;
  a.count = 3; a.len = n_;
  dots_async(a, part_r, 0);
  DotSpec b{};  // m-length: |y/Dl|_inf, |dy/Dl|_inf, h'(dy/Dl)
  b.a[0] = y; b.sa[0] = Dl; b.kind[0] = DK_MAXABS;
  b.a[1] = dys; b.sa[1] = Dl; b.kind[1] = DK_MAXABS;
  b.a[2] = h_raw; b.b[2] = dys; b.sa[2] = Dl; b.kind[2] = DK_DOT;
  b.count = 3; b.len = m_;
  dots_async(b, part_x, 3);
  OpResidual opp{gd, Dl, 1.0, nullptr, 0.0, h_raw, tm[5], bl_fin, bu_fin, 0};
  finalize_async(part_a, launch_project(opp, CON, part_a), 7, 0b0010110u, 6);
  OpResidual opd{ad, Dr, -1.0, c_raw, 1.0, nullptr, tn[5], bl_fin, bu_fin, nb_};
  finalize_async(part_b, launch_project(opd, SLK, part_b), 7, 0b0010110u, 13);
  const double* r = fetch(20);
  {
    Infea& I = ii[0];
    I.primal_ray_obj = ci[0].pobj;
    I.dual_ray_obj = ci[0].dobj;
    I.max_primal_ray_inf = (ci[0].pobj < 0.0) ? ci[0].linf_abs_p : 1e10;
    I.max_dual_ray_inf = (ci[0].dobj > 0.0) ? ci[0].linf_abs_d : 1e10;
    I.primal_ray_norm = r[0];
    I.dual_ray_norm = r[3];
    push_trend(I);
  }
  {
    Infea& I = ii[1];
    double pobj = r[2];
    double dobj = r[5] + r[13 + 6];
    I.primal_ray_obj = pobj;
    I.dual_ray_obj = dobj;
    I.max_primal_ray_inf = (pobj < 0.0) ? r[6 + 1] : 1e10;
    I.max_dual_ray_inf = (dobj > 0.0) ? r[13 + 1] : 1e10;
    I.primal_ray_norm = r[1];
    I.dual_ray_norm = r[4];
    push_trend(I);
  }
  check_termination();
}

// check_termination_criteria (src/pdcs_gpu/termination.jl:74-260) on the
// current (ci[0], ii[0]) and averaged (ci[1], ii[1]) sequences; sets
// exit_code (PDCS_EXIT_CONTINUE while running), the reported objectives and
// which sequence is returned.
static void termination_check(Converge (&ci)[2], Infea (&ii)[2], int64_t iter, const pdcs_options& O,
                              double elapsed, int& exit_code_, double& pobj_, double& dobj_, int& returned_seq_) {
  auto mono = [](const std::vector<double>& b, bool inc) {
    if (b.size() < 20) return false;
    for (size_t i = 1; i < 20; ++i)
      if (inc ? (b[i] < b[i - 1]) : (b[i] > b[i - 1])) return false;
    return true;
  };
  for (int k = 0; k < 2; ++k) {
    Converge& C = ci[k];
    if (std::max(C.linf_rel_p, std::max(C.linf_rel_d, C.rel_gap)) < O.rel_tol) C.status = PDCS_EXIT_OPTIMAL;
    if (std::max(C.linf_abs_p, std::max(C.linf_abs_d, C.abs_gap)) < O.abs_tol) C.status = PDCS_EXIT_OPTIMAL;
    if (std::isnan(C.rel_gap)) C.status = PDCS_EXIT_NUMERICAL_NAN;
    if (std::isinf(C.rel_gap)) C.status = PDCS_EXIT_NUMERICAL_INF;
    if (C.status == PDCS_EXIT_OPTIMAL) {
      exit_code_ = PDCS_EXIT_OPTIMAL;
      pobj_ = C.pobj;
      dobj_ = C.dobj;
      returned_seq_ = k;
      return;
    }
    if (C.status == PDCS_EXIT_NUMERICAL_NAN || C.status == PDCS_EXIT_NUMERICAL_INF) {
      exit_code_ = C.status;
      return;
    }
  }
  for (int k = 0; k < 2; ++k) {
    Infea& I = ii[k];
    if (I.dual_ray_obj > 0.0) {
      if ((I.dual_ray_obj - I.primal_ray_obj) / (1 + std::fabs(I.dual_ray_obj) + std::fabs(I.primal_ray_obj)) > 0.99999 &&
          I.max_primal_ray_inf > 1e3 && mono(I.dtrend, true) && I.max_dual_ray_inf > 1e4 && I.dual_ray_obj > 1e14 &&
          I.dual_ray_norm > 1e8)
        I.status = PDCS_EXIT_PRIMAL_INFEASIBLE_LOW_ACC;
      double res = std::max(I.max_dual_ray_inf, 1.0) / I.dual_ray_obj;
      if (res <= O.eps_primal_infeasible_low_acc) {
        if (res <= O.eps_primal_infeasible_high_acc) I.status = PDCS_EXIT_PRIMAL_INFEASIBLE_HIGH_ACC;
        if (I.max_dual_ray_inf > 1e8) I.status = PDCS_EXIT_PRIMAL_INFEASIBLE_LOW_ACC;
        if (mono(I.dtrend, true)) I.status = PDCS_EXIT_PRIMAL_INFEASIBLE_LOW_ACC;
      }
    }
    if ((I.status == 2 && iter > 2000) || (I.status == 3 && iter > 500)) {
      exit_code_ = I.status;
      pobj_ = I.primal_ray_obj;
      dobj_ = I.dual_ray_obj;
      return;
    }
    if (I.primal_ray_obj < 0.0) {
      if ((I.primal_ray_obj - I.dual_ray_obj) / (1 + std::fabs(I.primal_ray_obj) + std::fabs(I.dual_ray_obj)) > 0.99999 &&
          I.max_dual_ray_inf > 1e3 && mono(I.ptrend, false) && I.max_primal_ray_inf > 1e4 &&
          -I.primal_ray_obj > 1e14 && I.primal_ray_norm > 1e8)
        I.status = PDCS_EXIT_DUAL_INFEASIBLE_LOW_ACC;
      double res = std::max(I.max_primal_ray_inf, 1.0) / (-I.primal_ray_obj);
      if (res <= O.eps_dual_infeasible_low_acc) {
        if (res <= O.eps_dual_infeasible_high_acc) I.status = PDCS_EXIT_DUAL_INFEASIBLE_HIGH_ACC;
        if (I.max_primal_ray_inf > 1e8) I.status = PDCS_EXIT_DUAL_INFEASIBLE_LOW_ACC;
        if (mono(I.ptrend, false)) I.status = PDCS_EXIT_DUAL_INFEASIBLE_LOW_ACC;
      }
    }
    if ((I.status == 4 && iter > 2000) || (I.status == 5 && iter > 500)) {
      exit_code_ = I.status;
      pobj_ = I.primal_ray_obj;
      dobj_ = I.dual_ray_obj;
      return;
    }
  }
  if ((double)iter >= (double)O.max_outer_iter * (double)O.max_inner_iter) {
    exit_code_ = PDCS_EXIT_MAX_ITER;
    pobj_ = ci[0].pobj;
    dobj_ = ci[0].dobj;
    return;
  }
  if (O.time_limit > 0 && elapsed > O.time_limit) {
    exit_code_ = PDCS_EXIT_TIME_LIMIT;
    return;
  }
  exit_code_ = PDCS_EXIT_CONTINUE;
}

void Solver::check_termination() {
  termination_check(ci, ii, S.iter, O, now_s() - t_start_, exit_code_, pobj_, dobj_, returned_seq_);
}

// Mnorm (rpdhg_alg_gpu_gen.jl:133-138)
double Solver::mnorm(const double* dx, const double* dy, double ta, double si) {
  double* gdx = tm[4];
  spmv(G_, dx, gdx);
  DotSpec d{};  // m-length: y'Gx, y'y
  d.a[0] = dy; d.b[0] = gdx; d.kind[0] = DK_DOT;
  d.a[1] = dy; d.kind[1] = DK_DOT;
  d.count = 2; d.len = m_;
  dots_async(d, part_r, 0);
  DotSpec e{};
  e.a[0] = dx; e.kind[0] = DK_DOT;
  e.count = 1; e.len = n_;
  dots_async(e, part_x, 2);
  const double* r = fetch(3);
  return r[2] / ta - 2.0 * r[0] + r[1] / si;
}

// binary_search_duality_gap_diagonal! (rpdhg_alg_gpu_gen_scaling.jl:20-117);
// the doubling loop's `tRight = t, tLeft = t / 2, break` parses as
// `tRight = ((t, tLeft) = (t / 2, break))`, i.e. a plain break.
double Solver::binary_search(double r, const double* px, const double* py, double ta, double si) {
  double* h1 = tn[2];
  double* h2 = tm[2];
  double* xs = tn[3];
  double* ys = tm[3];
  double* gpx = tm[1];
  double* gxs = tm[4];
  spmv(Gt_, py, h1);
  axpby(h1, 1.0, h1, -1.0, c_s, n_);
  spmv(G_, px, gpx);
  axpby(h2, -1.0, gpx, 1.0, h_s, m_);
  double last_h1dx = 0.0, last_h2dy = 0.0;
  auto approx = [&](double t) {
    probes_++;
    OpAxpyProj ox{px, h1, t * ta / 2, xs, nullptr, nullptr};
    finalize_async(part_a, launch_project(ox, XI, part_a), 3, 0u, 0);
    spmv(G_, xs, gxs);
    OpAxpyProj oy{py, h2, t * si / 2, ys, gxs, gpx};
    finalize_async(part_b, launch_project(oy, YI, part_b), 3, 0u, 3);
    const double* r = fetch(6);
    last_h1dx = r[1];
    last_h2dy = r[4];
    return r[0] / ta - 2.0 * r[5] + r[3] / si;
  };
  double t = bs_t0_, tR = t, tL = 0.0;
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
  bs_t0_ = tM;
  return (last_h1dx + last_h2dy) / r;
}

// restart_threshold_calculation_diagonal! (rpdhg_alg_gpu_gen_scaling.jl:354-393)
void Solver::restart_threshold(bool dgap) {
  Timer tm_(t_restart_);
  if (dgap) {
    double* dx = tn[4];
    double* dy = tm[5];
    axpby(dx, 1.0, x0, -1.0, x0l, n_);
    axpby(dy, 1.0, y0, -1.0, y0l, m_);
    double r = mnorm(dx, dy, S.tau, S.sigma);
    ndg_r_ = r;
    ndg_thr_ = binary_search(r, x0, y0, S.tau, S.sigma);
    if (ndg_thr_ < 0) dgap_flag_ = false;
  } else {
    converge_info(x, y, ci[0], tm[0], tn[0]);
    kkt_thr_ = kkt_error(ci[0]);
  }
}

// restart_condition_check_diagonal! (rpdhg_alg_gpu_gen_scaling.jl:395-506)
bool Solver::restart_check(bool dgap) {
  Timer tm_(t_restart_);
  auto to_current = [&]() {
    copy(xm, x, n_);
    copy(ym, y, m_);
  };
  if (dgap) {
    double* dx = tn[4];
    double* dy = tm[5];
    axpby(dx, 1.0, x, -1.0, x0, n_);
    axpby(dy, 1.0, y, -1.0, y0, m_);
    double rl = mnorm(dx, dy, S.tau, S.sigma);
    double rho = binary_search(rl, x, y, S.tau, S.sigma);
    double rho_m = binary_search(rl, xm, ym, S.tau, S.sigma);
    ndg_[0] = rho;
    ndg_[1] = rho_m;
    for (double beta : {0.4, 0.8}) {
      if (rho < beta * ndg_thr_ || rho_m < beta * ndg_thr_) {
        restart_used_++;
        if (ndg_[0] < ndg_[1] && dgap_flag_) to_current();
        return true;
      }
    }
  } else {
    converge_info(x, y, ci[0], tm[0], tn[0]);
    converge_info(xm, ym, ci[1], tm[1], tn[1]);
    double lag0 = kkt_err_[0], lag1 = kkt_err_[1];
    double e0 = kkt_error(ci[0]), e1 = kkt_error(ci[1]);
    kkt_err_[0] = e0;
    kkt_err_[1] = e1;
    bool c1 = e0 < 0.4 * kkt_thr_ || e1 < 0.4 * kkt_thr_;
    bool c2 = (e0 < 0.8 * kkt_thr_ && e0 > lag0) || (e1 < 0.8 * kkt_thr_ && e1 > lag1);
    if (c1 || c2) {
      restart_used_++;
      if (kkt_err_[0] < kkt_err_[1]) to_current();
      return true;
    }
  }
  if ((double)S.inner >= (double)S.iter * 0.223 && S.iter > 100000) {
    restart_used_++;
    return true;
  }
  return false;
}

void Solver::run_until_halt() {
  Timer tm_(t_iter_);
  push_state();
  if (!graph_exec_) capture_graph();
  if (fp32_) anchor(nullptr, nullptr, nullptr);
  while (true) {
    int64_t to_check = S.check_freq > 0 ? S.check_freq - (S.iter % S.check_freq) : 1 << 20;
    int64_t graphs = (to_check + attempts_per_graph_ - 1) / attempts_per_graph_;
    graphs = std::max<int64_t>(1, std::min<int64_t>(graphs, 4));
    for (int64_t g = 0; g < graphs; ++g) {
      PDCS_CUDA(cudaGraphLaunch(graph_exec_, s_));
      graphs_++;
      kernels_ += 5LL * attempts_per_graph_;
    }
    pull_state();
    if (!S.active) break;
    if (O.time_limit > 0 && now_s() - t_start_ > O.time_limit) break;
    if (fp32_) {  // FP64 refinement: new anchors, so the FP32 deltas stay one round's movement
      materialize(nullptr, nullptr, nullptr);
      anchor(nullptr, nullptr, nullptr);
    }
  }
  if (fp32_) materialize(nullptr, nullptr, nullptr);  // the host works on the FP64 iterates
}

void Solver::log_progress() {
  if (!O.verbose) return;
  std::printf("[pdcs_b200] iter %lld rel_p %.3e rel_d %.3e gap %.3e pobj %.8e dobj %.8e restarts %lld time %.3f\n",
              (long long)S.iter, ci[0].linf_rel_p, ci[0].linf_rel_d, ci[0].rel_gap, ci[0].pobj, ci[0].dobj,
              (long long)restart_used_, now_s() - t_start_);
}

// pdhg_main_iter_average_diagonal_rescaling_restarts_adaptive_weight_resolving_aggressive!
// (rpdhg_alg_gpu_gen_scaling.jl:770-895)
void Solver::main_loop() {
  copy(x0, x, n_);
  copy(y0, y, m_);
  copy(x0l, x, n_);
  copy(y0l, y, m_);
  S = PdhgState{};
  S.omega = init_omega();
  S.eta_p = 1.0 / ginf_;
  S.tau = 0.9;
  S.sigma = 0.9;
  S.check_freq = O.check_terminate_freq;
  S.attempt_limit = O.attempt_limit;
  // one restart frequency drives the device halt; both restart tests run on the host
  int64_t rf = 0;
  if (O.use_duality_gap_restart) rf = O.duality_gap_restart_freq;
  if (O.use_kkt_restart) rf = rf ? std::min(rf, O.kkt_restart_freq) : O.kkt_restart_freq;
  S.restart_freq = rf;
  S.restart_enabled = rf > 0;
  for (int64_t outer = 1; outer <= O.max_outer_iter; ++outer) {
    // update_best_sol! (:640-649)
    if (ci[0].l2_rel_p < pres_best_) { pres_best_ = ci[0].l2_rel_p; copy(xbest, x, n_); }
    if (ci[0].l2_rel_d < dres_best_) { dres_best_ = ci[0].l2_rel_d; copy(ybest, y, m_); }
    max_kkt_ = std::max(std::max(ci[0].l2_rel_p, ci[0].l2_rel_d), ci[0].rel_gap);
    min_kkt_ = std::min(std::min(std::min(ci[0].l2_rel_p, ci[0].l2_rel_d), ci[0].rel_gap), min_kkt_);
    double extra = -0.1 * std::log10(max_kkt_) + 0.2;
    copy(x0l, x0, n_);
    copy(y0l, y0, m_);
    copy(x0, xm, n_);
    copy(y0, ym, m_);
    copy(x, xm, n_);
    copy(y, ym, m_);
    if (O.use_kkt_restart) restart_threshold(false);
    else restart_threshold(dgap_flag_);
    // resolving triggers (:810-838)
    {
      double pd = ci[0].l2_rel_p / ci[0].l2_rel_d;
      bool f1 = outer > 10 && max_kkt_ > 1e5;
      bool f2 = outer > 80 && (pd > 1e10 || pd < 1e-10);
      bool f3 = outer > 10 && S.tau < 1e-6 && S.sigma < 1e-6;
      bool f4 = S.iter > 1000000 && ci[0].rel_gap > 0.98 && ci[0].l2_rel_p > 1.0 && ci[0].l2_rel_d > 1.0;
      if (f1 || f2 || f3 || f4 || O.force_resolving) {
        if (O.verbose) std::printf("[pdcs_b200] resolving fallback at outer %lld\n", (long long)outer);
        resolving();
        return;
      }
    }
    double* xds = xds_;
    double* yds = yds_;
    copy(xl, x, n_);
    copy(yl, y, m_);
    copy(xds, x, n_);
    copy(yds, y, m_);
    // start of the inner loop (:839-842) and of the first step call (:667, :676)
    S.inner = 0;
    S.eta_cum = 0.0;
    S.extra = extra;
    S.dec = decay(max_kkt_);
    S.dec_next = S.dec;
    S.eta = std::max(S.eta_p, 1e-6);
    S.reject_count = 0;
    S.ps = (S.eta / S.omega) * S.dec;
    S.ds = (S.eta * S.omega) * S.dec;
    S.active = 1;
    S.halt_reason = HALT_NONE;
    S.do_reflect = 0;
    bool restart = false;
    while (!restart) {
      run_until_halt();
      if (O.time_limit > 0 && now_s() - t_start_ > O.time_limit && S.active) {
        exit_code_ = PDCS_EXIT_TIME_LIMIT;
        return;
      }
      int reason = S.halt_reason;
      S.halt_reason = HALT_NONE;
      if (reason == HALT_LIMIT) {
        exit_code_ = PDCS_EXIT_ATTEMPT_LIMIT;
        return;
      }
      if (reason == HALT_CHECK) {
        exit_check();
        max_kkt_ = std::max(std::max(ci[0].l2_rel_p, ci[0].l2_rel_d), ci[0].rel_gap);
        S.dec_next = decay(max_kkt_);
        log_progress();
        if (exit_code_ != PDCS_EXIT_CONTINUE) return;
        if (S.attempt_limit > 0 && S.iter >= S.attempt_limit) {
          exit_code_ = PDCS_EXIT_ATTEMPT_LIMIT;
          return;
        }
        if (S.accepted) {
          post_accept(S, false);
        } else {
          after_reject(S);
          if (S.reject_count > 1000000) {
            S.eta = S.eta_p;
            post_accept(S, true);
          }
        }
        if (S.do_reflect) {
          push_state();
          reflect_kernel<<<grid_reflect_, kThreads, 0, s_>>>(st_dev, x, xl, xm, n_, y, yl, ym, m_);
          kernels_++;
          S.do_reflect = 0;
        }
        reason = S.halt_reason;
        S.halt_reason = HALT_NONE;
        if (reason == HALT_NONE) {
          S.active = 1;
          continue;
        }
      }
      if (reason == HALT_ARTIFICIAL) {
        restart_used_++;
        restart = true;
        break;
      }
      if (reason == HALT_RESTART_CHECK) {
        bool brk = false;
        if (O.use_kkt_restart && O.kkt_restart_freq > 0 && S.iter % O.kkt_restart_freq == 0) {
          if (restart_check(false) || outer == 1) brk = true;
        }
        if (!brk && O.use_duality_gap_restart && O.duality_gap_restart_freq > 0 &&
            S.iter % O.duality_gap_restart_freq == 0) {
          if (restart_check(dgap_flag_) || outer == 1) brk = true;
        }
        if (brk) {
          restart = true;
          break;
        }
        S.active = 1;
        continue;
      }
    }
    omega_update(xds, yds, false);
  }
  exit_code_ = PDCS_EXIT_MAX_ITER;
}

// dynamic_primal_weight_update (rpdhg_alg_gpu_gen_scaling.jl:284-307); the
// resolving loop clamps the result to [0.8, 1.2] (:632-633)
void Solver::omega_update(double* xds, double* yds, bool clamp) {
  DotSpec d{};
  d.a[0] = xds; d.b[0] = x; d.kind[0] = DK_DIFF2;
  d.count = 1; d.len = n_;
  double xn2;
  dots(d, &xn2);
  DotSpec e{};
  e.a[0] = yds; e.b[0] = y; e.kind[0] = DK_DIFF2;
  e.count = 1; e.len = m_;
  double yn2;
  dots(e, &yn2);
  double xn = std::sqrt(xn2), yn = std::sqrt(yn2), om = S.omega;
  if ((om > 1e4 || om < 1e-4) && restart_used_ % 20 == 0 && restart_used_ != 0) S.omega = init_omega();
  else if ((om > 3e4 || om < 1.0 / 3e4) && restart_used_ % 10 == 0 && restart_used_ != 0) S.omega = init_omega();
  else if (xn > 1e-10 && yn > 1e-10) S.omega = std::exp(0.5 * std::log(yn / xn) + 0.5 * std::log(om));
  if (clamp) S.omega = std::min(std::max(S.omega, 0.8), 1.2);
}

// power_method! (def_rpdhg_gen.jl:891-917): sqrt of the largest eigenvalue of
// G'G (scaled G), tolerance 1e-3, at most 1000 iterations; the start vector
// is a fixed pseudo-random sequence (the reference draws rand(n)).
double Solver::power_method(bool* converged) {
  std::vector<double> b0(n_);
  uint64_t st = 0x9E3779B97F4A7C15ull;
  for (int64_t j = 0; j < n_; ++j) {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    b0[j] = (double)(st >> 11) * (1.0 / 9007199254740992.0);
  }
  double* b = tn[0];
  double* ab = tm[0];
  double* atab = tn[1];
  PDCS_CUDA(cudaMemcpyAsync(b, b0.data(), sizeof(double) * n_, cudaMemcpyHostToDevice, s_));
  double nb = nrm2(b, n_);
  axpby(b, 1.0 / nb, b, 0.0, nullptr, n_);
  double lam_old = 0.0, lam = 0.0;
  for (int it = 0; it < 1000; ++it) {
    spmv(G_, b, ab);
    spmv(Gt_, ab, atab);
    nb = nrm2(atab, n_);
    axpby(b, 1.0 / nb, atab, 0.0, nullptr, n_);
    spmv(G_, b, ab);
    spmv(Gt_, ab, atab);
    DotSpec d{};
    d.a[0] = b; d.b[0] = atab; d.kind[0] = DK_DOT;
    d.count = 1; d.len = n_;
    dots(d, &lam);
    if (std::fabs(lam - lam_old) < 1e-3) {
      *converged = true;
      return std::sqrt(lam);
    }
    lam_old = lam;
  }
  *converged = false;
  return std::sqrt(lam);
}

// resolving_pessimistic_step! (rpdhg_alg_gpu_gen_scaling.jl:511-638)
void Solver::resolving() {
  bool conv = false;
  double gl = power_method(&conv);
  double step = (conv ? 0.9 : 0.8) / gl;
  S.tau = step;
  S.sigma = step;
  S.omega = std::min(std::max(init_omega(), 0.8), 1.2);
  copy(xm, xbest, n_);
  copy(ym, ybest, m_);
  for (int64_t outer = 1; outer <= O.max_outer_iter; ++outer) {
    copy(x0l, x0, n_);
    copy(y0l, y0, m_);
    copy(x0, xm, n_);
    copy(y0, ym, m_);
    copy(x, xm, n_);
    copy(y, ym, m_);
    if (O.use_kkt_restart) restart_threshold(false);
    else restart_threshold(dgap_flag_);
    copy(xl, x, n_);
    copy(yl, y, m_);
    copy(xds_, x, n_);
    copy(yds_, y, m_);
    S.resolving = 1;
    S.inner = 0;
    S.ps = S.tau / S.omega;
    S.ds = S.sigma * S.omega;
    S.eta = 1.0;  // unused by the fixed-step control
    S.active = 1;
    S.halt_reason = HALT_NONE;
    S.do_reflect = 0;
    while (true) {
      run_until_halt();
      if (O.time_limit > 0 && now_s() - t_start_ > O.time_limit && S.active) {
        exit_code_ = PDCS_EXIT_TIME_LIMIT;
        return;
      }
      int reason = S.halt_reason;
      S.halt_reason = HALT_NONE;
      if (reason == HALT_LIMIT) {
        exit_code_ = PDCS_EXIT_ATTEMPT_LIMIT;
        return;
      }
      // :570-596: the restart tests come first and break before the exit check
      bool brk = false;
      if (O.use_kkt_restart && O.kkt_restart_freq > 0 && S.iter % O.kkt_restart_freq == 0)
        if (restart_check(false) || outer == 1) brk = true;
      if (!brk && O.use_duality_gap_restart && O.duality_gap_restart_freq > 0 &&
          S.iter % O.duality_gap_restart_freq == 0)
        if (restart_check(dgap_flag_) || outer == 1) brk = true;
      if (brk) break;
      if (O.check_terminate_freq > 0 && S.iter % O.check_terminate_freq == 0) {
        exit_check();
        log_progress();
        if (exit_code_ != PDCS_EXIT_CONTINUE) return;
      }
      if (S.attempt_limit > 0 && S.iter >= S.attempt_limit) {
        exit_code_ = PDCS_EXIT_ATTEMPT_LIMIT;
        return;
      }
      S.active = 1;
    }
    omega_update(xds_, yds_, true);
  }
  exit_code_ = PDCS_EXIT_MAX_ITER;
}

int Solver::run(pdcs_result* res) {
  int rc = validate();
  if (rc != PDCS_OK) return rc;
  double t0 = now_s();
  setup();
  converge_info(x, y, ci[0], tm[0], tn[0]);  // rpdhg_alg_gpu_gen.jl:1865-1881
  t_start_ = now_s();
  res->setup_time = t_start_ - t0;
  main_loop();
  PDCS_CUDA(cudaStreamSynchronize(s_));
  res->time = now_s() - t_start_;
  const bool mean = (exit_code_ == PDCS_EXIT_OPTIMAL && returned_seq_ == 1);
  double* xo = tn[0];
  double* yo = tm[0];
  div_kernel<<<grid_for(n_), kThreads, 0, s_>>>(xo, mean ? xm : x, Dr, n_);
  div_kernel<<<grid_for(m_), kThreads, 0, s_>>>(yo, mean ? ym : y, Dl, m_);
  if (res->x) PDCS_CUDA(cudaMemcpyAsync(res->x, xo, sizeof(double) * n_, cudaMemcpyDeviceToHost, s_));
  if (res->y) PDCS_CUDA(cudaMemcpyAsync(res->y, yo, sizeof(double) * m_, cudaMemcpyDeviceToHost, s_));
  if (res->x_device) PDCS_CUDA(cudaMemcpyAsync(res->x_device, xo, sizeof(double) * n_, cudaMemcpyDeviceToDevice, s_));
  if (res->y_device) PDCS_CUDA(cudaMemcpyAsync(res->y_device, yo, sizeof(double) * m_, cudaMemcpyDeviceToDevice, s_));
  PDCS_CUDA(cudaStreamSynchronize(s_));
  const Converge& C = ci[mean ? 1 : 0];
  res->exit_code = exit_code_;
  res->returned_sequence = mean ? 1 : 0;
  res->pObj = (exit_code_ == PDCS_EXIT_OPTIMAL || exit_code_ == PDCS_EXIT_MAX_ITER) ? C.pobj : pobj_;
  res->dObj = (exit_code_ == PDCS_EXIT_OPTIMAL || exit_code_ == PDCS_EXIT_MAX_ITER) ? C.dobj : dobj_;
  res->iter = S.iter;
  res->restart_used = restart_used_;
  res->l_inf_rel_primal_res = C.linf_rel_p;
  res->l_inf_rel_dual_res = C.linf_rel_d;
  res->rel_gap = C.rel_gap;
  res->l_2_rel_primal_res = C.l2_rel_p;
  res->l_2_rel_dual_res = C.l2_rel_d;
  res->l_inf_abs_primal_res = C.linf_abs_p;
  res->l_inf_abs_dual_res = C.linf_abs_d;
  res->abs_gap = C.abs_gap;
  res->kernel_launches = kernels_;
  res->graph_launches = graphs_;
  res->time_iterations = t_iter_;
  res->time_exit_checks = t_exit_;
  res->time_restarts = t_restart_;
  res->restart_probes = probes_;
  res->spmv_lane_nnz_G = lane_G_;
  res->spmv_lane_nnz_Gt = lane_Gt_;
  return PDCS_OK;
}

}  // namespace pdcs

#include "pdcs_batch.cuh"

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int pdcs_default_options(pdcs_options* o) {
  if (!o) return PDCS_ERR_INVALID;
  std::memset(o, 0, sizeof(*o));
  o->rescaling_method = 3;
  o->use_preconditioner = 1;
  o->use_adaptive_restart = 1;
  o->use_adaptive_step_size_weight = 1;
  o->use_aggressive = 1;
  o->use_accelerated = 0;
  o->use_resolving = 1;
  o->warm_start = 0;
  o->max_outer_iter = 10000;
  o->max_inner_iter = 500000;
  o->abs_tol = 1e-6;
  o->rel_tol = 1e-6;
  o->eps_primal_infeasible_low_acc = 1e-12;
  o->eps_dual_infeasible_low_acc = 1e-12;
  o->eps_primal_infeasible_high_acc = 1e-16;
  o->eps_dual_infeasible_high_acc = 1e-16;
  o->print_freq = 2000;
  o->check_terminate_freq = 2000;
  o->verbose = 0;
  o->use_kkt_restart = 0;
  o->time_limit = 0.0;
  o->kkt_restart_freq = 2000;
  o->use_duality_gap_restart = 1;
  o->precision = 0;
  o->duality_gap_restart_freq = 2000;
  o->attempt_limit = 0;
  o->stream = nullptr;
  o->attempts_per_graph = 32;
  return PDCS_OK;
}

int pdcs_solve(const pdcs_problem* prob, const pdcs_options* opts, pdcs_result* res) {
  if (!prob || !res) return PDCS_ERR_INVALID;
  pdcs_options o;
  if (opts) o = *opts;
  else pdcs_default_options(&o);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return PDCS_ERR_NO_DEVICE;
  try {
    pdcs::Solver s(prob, &o);
    const int rc = s.run(res);
    if (s.huge_failed()) {
      std::fprintf(stderr, "pdcs_solve: a cooperative projection of a huge cone timed out at a barrier\n");
      return PDCS_ERR_CUDA;
    }
    return rc;
  } catch (const pdcs::CudaError& e) {
    std::fprintf(stderr, "pdcs_solve: %s\n", e.what());
    return PDCS_ERR_CUDA;
  } catch (const std::domain_error&) {
    return PDCS_ERR_BOUNDS;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "pdcs_solve: %s\n", e.what());
    return PDCS_ERR_INVALID;
  }
}

int pdcs_solve_batch(int64_t count, const pdcs_problem* problems, const pdcs_options* opts, pdcs_result* results,
                     pdcs_batch_info* info) {
  if (count < 1 || !problems || !results) return PDCS_ERR_INVALID;
  pdcs_options o;
  if (opts) o = *opts;
  else pdcs_default_options(&o);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return PDCS_ERR_NO_DEVICE;
  try {
    pdcs::BatchSolver b(count, problems, &o);
    return b.run_batch(results, info);
  } catch (const pdcs::CudaError& e) {
    std::fprintf(stderr, "pdcs_solve_batch: %s\n", e.what());
    return PDCS_ERR_CUDA;
  } catch (const std::domain_error&) {
    return PDCS_ERR_BOUNDS;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "pdcs_solve_batch: %s\n", e.what());
    return PDCS_ERR_INVALID;
  }
}

struct pdcs_batch {
  pdcs::BatchSolver* solver;
};

int pdcs_batch_create(int64_t count, const pdcs_problem* problems, const pdcs_options* opts, pdcs_batch** out) {
  if (count < 1 || !problems || !out) return PDCS_ERR_INVALID;
  *out = nullptr;
  pdcs_options o;
  if (opts) o = *opts;
  else pdcs_default_options(&o);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return PDCS_ERR_NO_DEVICE;
  pdcs::BatchSolver* b = nullptr;
  try {
    b = new pdcs::BatchSolver(count, problems, &o);
    int rc = b->prepare();
    if (rc != PDCS_OK) {
      delete b;
      return rc;
    }
    *out = new pdcs_batch{b};
    return PDCS_OK;
  } catch (const pdcs::CudaError& e) {
    std::fprintf(stderr, "pdcs_batch_create: %s\n", e.what());
    delete b;
    return PDCS_ERR_CUDA;
  } catch (const std::domain_error&) {
    delete b;
    return PDCS_ERR_BOUNDS;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "pdcs_batch_create: %s\n", e.what());
    delete b;
    return PDCS_ERR_INVALID;
  }
}

int pdcs_batch_solve(pdcs_batch* batch, int64_t attempt_limit, pdcs_result* results, pdcs_batch_info* info) {
  if (!batch || !batch->solver || !results) return PDCS_ERR_INVALID;
  try {
    return batch->solver->solve(results, info, attempt_limit);
  } catch (const pdcs::CudaError& e) {
    std::fprintf(stderr, "pdcs_batch_solve: %s\n", e.what());
    return PDCS_ERR_CUDA;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "pdcs_batch_solve: %s\n", e.what());
    return PDCS_ERR_INVALID;
  }
}

static pdcs_grad_options grad_defaults(const pdcs_grad_options* g) {
  pdcs_grad_options o{};
  if (g) o = *g;
  if (o.rel_tol <= 0) o.rel_tol = 1e-10;
  if (o.restart <= 0) o.restart = 100;
  if (o.max_iter <= 0) o.max_iter = 5000;
  return o;
}

int pdcs_batch_grad(pdcs_batch* batch, const double* const* dldx, const double* const* dldy, double* const* dc,
                    double* const* dh, double* const* dG, double* const* dl, double* const* du,
                    const pdcs_grad_options* opts, pdcs_grad_info* info) {
  if (!batch || !batch->solver) return PDCS_ERR_INVALID;
  try {
    return batch->solver->grad(dldx, dldy, dc, dh, dG, dl, du, grad_defaults(opts), info);
  } catch (const pdcs::CudaError& e) {
    std::fprintf(stderr, "pdcs_batch_grad: %s\n", e.what());
    return PDCS_ERR_CUDA;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "pdcs_batch_grad: %s\n", e.what());
    return PDCS_ERR_INVALID;
  }
}

int pdcs_grad(const pdcs_problem* prob, const pdcs_options* opts, const double* x, const double* y,
              const double* dldx, const double* dldy, double* dc, double* dh, double* dG, double* dl, double* du,
              const pdcs_grad_options* gopts, pdcs_grad_info* info) {
  if (!prob || !x || !y) return PDCS_ERR_INVALID;
  pdcs_options o;
  if (opts) o = *opts;
  else pdcs_default_options(&o);
  o.differentiable = 1;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return PDCS_ERR_NO_DEVICE;
  try {
    pdcs::BatchSolver b(1, prob, &o);
    int rc = b.prepare();
    if (rc != PDCS_OK) return rc;
    b.set_solution(&x, &y);
    return b.grad(&dldx, &dldy, &dc, &dh, &dG, &dl, &du, grad_defaults(gopts), info);
  } catch (const pdcs::CudaError& e) {
    std::fprintf(stderr, "pdcs_grad: %s\n", e.what());
    return PDCS_ERR_CUDA;
  } catch (const std::domain_error&) {
    return PDCS_ERR_BOUNDS;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "pdcs_grad: %s\n", e.what());
    return PDCS_ERR_INVALID;
  }
}

void pdcs_batch_destroy(pdcs_batch* batch) {
  if (!batch) return;
  delete batch->solver;
  delete batch;
}

int pdcs_block_proj(double* arr, const double* bl, const double* bu, const double* S, const int64_t* head_start,
                    const int64_t* ns, int64_t blkNum, const int64_t* proj_type, void* stream) {
  if (blkNum < 0) return PDCS_ERR_INVALID;
  if (blkNum == 0) return PDCS_OK;
  if (!arr || !head_start || !ns || !proj_type) return PDCS_ERR_INVALID;
  int64_t grid = std::min<int64_t>((blkNum + pdcs::kWarps - 1) / pdcs::kWarps, 148 * 16);
  pdcs::block_proj_kernel<<<(int)grid, pdcs::kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      arr, bl, bu, S, head_start, ns, blkNum, proj_type);
  return cudaGetLastError() == cudaSuccess ? PDCS_OK : PDCS_ERR_CUDA;
}

int pdcs_spmv_csr(int64_t m, int64_t n, int64_t nnz, const int32_t* rowptr, const int32_t* colind, const double* val,
                  const double* x, double* y, void* stream) {
  if (m < 0 || n < 0 || nnz < 0) return PDCS_ERR_INVALID;
  if (m == 0) return PDCS_OK;
  if (!rowptr || !y || (nnz > 0 && (!colind || !val || !x))) return PDCS_ERR_INVALID;
  if (m > INT32_MAX || nnz > INT32_MAX) return PDCS_ERR_INVALID;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t nctas = (m + nnz + pdcs::kMergeItems - 1) / pdcs::kMergeItems;
  if (nctas > INT32_MAX) return PDCS_ERR_INVALID;
  // workspace for the per-CTA row carries (stream-ordered, like cuSPARSE's SpMV buffer)
  void* ws = nullptr;
  const size_t carry_bytes = ((size_t)nctas * sizeof(double) + 255) & ~(size_t)255;
  if (cudaMallocAsync(&ws, carry_bytes + (size_t)nctas * sizeof(int32_t), s) != cudaSuccess) return PDCS_ERR_CUDA;
  double* carry_val = static_cast<double*>(ws);
  int32_t* carry_row = reinterpret_cast<int32_t*>(static_cast<char*>(ws) + carry_bytes);
  pdcs::spmv_merge_kernel<<<(unsigned)nctas, pdcs::kThreads, 0, s>>>(m, nnz, rowptr, colind, val, x, y, carry_row,
                                                                   carry_val);
  int fg = (int)std::min<int64_t>((nctas + pdcs::kThreads - 1) / pdcs::kThreads, 148 * 8);
  pdcs::spmv_merge_fixup_kernel<<<fg, pdcs::kThreads, 0, s>>>(nctas, carry_row, carry_val, y);
  cudaError_t e = cudaGetLastError();
  if (cudaFreeAsync(ws, s) != cudaSuccess) return PDCS_ERR_CUDA;
  return e == cudaSuccess ? PDCS_OK : PDCS_ERR_CUDA;
}

// ---------------------------------------------------------------------------
// pdcs_spmv_csr_noalloc: pdcs_spmv_csr for callers that cannot allocate
// device memory (see include/pdcs.h).  The per-CTA carries live in a
// file-scope device array, sized for kNoAllocMaxCtas CTAs: 65536 CTAs of
// 2048 merge items, i.e. m + nnz <= 134,217,728; 768 KiB that every GPU which
// loads this library holds until the process exits.
// ---------------------------------------------------------------------------
static constexpr int64_t kNoAllocMaxCtas = 65536;
static __device__ __align__(256) unsigned char g_spmv_noalloc_scratch[kNoAllocMaxCtas * (sizeof(double) + sizeof(int32_t))];

namespace {
constexpr int kNoAllocMaxDevices = 128;
std::mutex g_noalloc_mu;
struct NoAllocEntry {
  void* ctx;   // the context the address was looked up in
  void* addr;  // device address of g_spmv_noalloc_scratch in that context
};
NoAllocEntry g_noalloc[kNoAllocMaxDevices] = {};

// The calling thread's current context (cuCtxGetCurrent, reached through the
// runtime's driver entry-point table, so the library needs no -lcuda).
void* current_context() {
  using CtxGetCurrent = int (*)(void**);
  static CtxGetCurrent fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return static_cast<CtxGetCurrent>(nullptr);
    return reinterpret_cast<CtxGetCurrent>(p);
  }();
  void* ctx = nullptr;
  if (fn) fn(&ctx);
  return ctx;
}

// Device address of the scratch array for the current device.  In host code
// the array's name is only a host-side stand-in; the address comes from
// cudaGetSymbolAddress with the device current, once per device and context:
// a context destroyed and recreated (cudaDeviceReset, a host runtime's device
// reset) gets a fresh lookup instead of a stale address.
int noalloc_scratch(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return PDCS_ERR_CUDA;
  if (dev < 0 || dev >= kNoAllocMaxDevices) return PDCS_ERR_INVALID;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoAllocEntry& e = g_noalloc[dev];
  void* ctx = current_context();
  if (!e.addr || !ctx || e.ctx != ctx) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_spmv_noalloc_scratch) != cudaSuccess || !p) return PDCS_ERR_CUDA;
    e.addr = p;
    e.ctx = current_context();  // the lookup makes the primary context current if none was
  }
  *out = e.addr;
  return PDCS_OK;
}
}  // namespace

int pdcs_spmv_csr_noalloc(int64_t m, int64_t n, int64_t nnz, const int32_t* rowptr, const int32_t* colind,
                          const double* val, const double* x, double* y, void* stream) {
  if (m < 0 || n < 0 || nnz < 0) return PDCS_ERR_INVALID;
  if (m == 0) return PDCS_OK;
  if (!rowptr || !y || (nnz > 0 && (!colind || !val || !x))) return PDCS_ERR_INVALID;
  if (m > INT32_MAX || nnz > INT32_MAX) return PDCS_ERR_INVALID;
  const int64_t nctas = (m + nnz + pdcs::kMergeItems - 1) / pdcs::kMergeItems;
  if (nctas > kNoAllocMaxCtas) return PDCS_ERR_NOALLOC_LIMIT;
  void* base = nullptr;
  int rc = noalloc_scratch(&base);
  if (rc != PDCS_OK) return rc;
  // every CTA writes its own carry entry, so nothing needs clearing between calls
  double* carry_val = static_cast<double*>(base);
  int32_t* carry_row = reinterpret_cast<int32_t*>(static_cast<char*>(base) + kNoAllocMaxCtas * sizeof(double));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  pdcs::spmv_merge_kernel<<<(unsigned)nctas, pdcs::kThreads, 0, s>>>(m, nnz, rowptr, colind, val, x, y, carry_row,
                                                                   carry_val);
  int fg = (int)std::min<int64_t>((nctas + pdcs::kThreads - 1) / pdcs::kThreads, 148 * 8);
  pdcs::spmv_merge_fixup_kernel<<<fg, pdcs::kThreads, 0, s>>>(nctas, carry_row, carry_val, y);
  return cudaGetLastError() == cudaSuccess ? PDCS_OK : PDCS_ERR_CUDA;
}

const char* pdcs_version(void) { return "pdcs_b200 0.1.0 (sm_100a, FP64)"; }

}  // extern "C"
