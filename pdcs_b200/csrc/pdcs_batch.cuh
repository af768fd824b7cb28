// pdcs_batch.cuh -- batched solver: many independent conic programs in one
// set of device launches, each with its own step sizes, restarts and
// termination.  Included by pdcs_solver.cu (it reuses the single-instance
// solver's setup, tables and helpers).
//
// Layout.  The K instances are merged into one block-diagonal program whose
// x and y are ordered by cone type across instances (x: all box parts, all
// SOC blocks, RSOC, exp, dual-exp; y: zero, nonneg, SOC, RSOC, exp,
// dual-exp).  The merged program is a valid single-instance problem, so the
// device preprocessing (Ruiz + Pock-Chambolle is row/column local, hence per
// instance), the binned SpMV and the cone tables are the single solver's.
//
// Control.  Each instance runs the reference's aggressive main loop
// (rpdhg_alg_gpu_gen_scaling.jl:770-895) as a C++ coroutine that suspends on
// every device request.  A scheduler groups the pending requests of all
// instances by kind and operands and runs each group as ONE masked launch
// sequence; instances that are iterating share CUDA graphs of PDHG attempts
// whose control kernel keeps every instance's eta / accept / halt state on
// the device.  Instances that reach their checkpoints at the same attempt
// (the common case) are serviced together.
#pragma once
#include <array>
#include <coroutine>
#include <exception>
#include <thread>
#include <type_traits>
#include <unordered_map>
#include <utility>

#include "pdcs_adjoint.cuh"
#include "pdcs_batch_kernels.cuh"
#include "pdcs_bsearch.cuh"
#include "pdcs_tiles.cuh"
#include "pdcs_fused.cuh"
#include "pdcs_tail.cuh"

namespace pdcs {

// ---------------------------------------------------------------------------
// Lazily started, awaitable coroutine returning T.
// ---------------------------------------------------------------------------
struct CoBase {
  std::coroutine_handle<> cont;
  std::exception_ptr ex;
  std::suspend_always initial_suspend() noexcept { return {}; }
  struct Final {
    bool await_ready() noexcept { return false; }
    template <class P>
    std::coroutine_handle<> await_suspend(std::coroutine_handle<P> h) noexcept {
      auto c = h.promise().cont;
      return c ? c : std::noop_coroutine();
    }
    void await_resume() noexcept {}
  };
  Final final_suspend() noexcept { return {}; }
  void unhandled_exception() { ex = std::current_exception(); }
};
template <class T>
struct CoPromise : CoBase {
  T value{};
  void return_value(T v) { value = std::move(v); }
};
template <>
struct CoPromise<void> : CoBase {
  void return_void() {}
};

template <class T = void>
class Co {
 public:
  struct promise_type : CoPromise<T> {
    Co get_return_object() { return Co(std::coroutine_handle<promise_type>::from_promise(*this)); }
  };
  Co() = default;
  explicit Co(std::coroutine_handle<promise_type> h) : h_(h) {}
  Co(Co&& o) noexcept : h_(std::exchange(o.h_, {})) {}
  Co& operator=(Co&& o) noexcept {
    if (this != &o) {
      if (h_) h_.destroy();
      h_ = std::exchange(o.h_, {});
    }
    return *this;
  }
  Co(const Co&) = delete;
  ~Co() {
    if (h_) h_.destroy();
  }
  bool await_ready() const noexcept { return false; }
  std::coroutine_handle<> await_suspend(std::coroutine_handle<> c) noexcept {
    h_.promise().cont = c;
    return h_;
  }
  T await_resume() {
    if (h_.promise().ex) std::rethrow_exception(h_.promise().ex);
    if constexpr (!std::is_void_v<T>) return std::move(h_.promise().value);
  }
  void start() { h_.resume(); }
  bool done() const { return !h_ || h_.done(); }
  void rethrow() const {
    if (h_ && h_.done() && h_.promise().ex) std::rethrow_exception(h_.promise().ex);
  }

 private:
  std::coroutine_handle<promise_type> h_;
};

// ---------------------------------------------------------------------------
// Device requests.  Requests whose payloads are byte-identical run as one
// batched operation over the union of the requesting instances.
// ---------------------------------------------------------------------------
enum ReqType : int32_t {
  RQ_NONE = 0,
  RQ_ITERATE,   // run PDHG attempts until this instance halts
  RQ_CONVERGE,  // KKT quantities of (p0, p1) -> out[0..15]; G p0 -> p2, G' p1 -> p3
  RQ_PROBE,     // one binary-search evaluation (restart duality gap)
  RQ_MNORM,     // G p0 -> p2; out = [p1'(G p0), p1'p1, p0'p0]
  RQ_SEG,       // per-instance reductions X / Y
  RQ_LIN,       // dst = a u + b v (up to 6, in order)
  RQ_SPMV,      // side 0: G p0 -> p1; side 1: G' p0 -> p1
  RQ_REFLECT,   // reflection + averaging with the instance's current coefficients
  RQ_BSEARCH,   // restart binary search(es) on the device: p0, p1 (then p2, p3); count searches
};

struct LinOp {
  double* dst;
  const double* u;
  const double* v;
  double a, b;
  int32_t side, pad;
};

struct ReqPayload {
  int32_t type, side, count, pad;
  const double* p[8];
  LinOp lin[6];
  SegSide X, Y;
};

struct Req {
  ReqPayload key;
  uint64_t hash = 0;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;  // per-instance scalars (probe steps, search parameters)
  double out[20] = {};
};

struct Inst {
  int64_t k = 0;
  PdhgState S{};
  Converge ci[2];
  Infea ii[2];
  int exit_code = PDCS_EXIT_CONTINUE;
  int returned_seq = 0;
  double pobj = 1e30, dobj = 1e30, max_kkt = 1e30, min_kkt = 1e30, pres_best = 1e30, dres_best = 1e30;
  double ndg[2] = {1e30, 1e30}, ndg_thr = 0, ndg_r = 1e30, kkt_err[2] = {1e30, 1e30}, kkt_thr = 0;
  bool dgap_flag = true;
  double bs_t0 = 1.0;
  int64_t restart_used = 0, check_count = 0, probes = 0;
  double hNrm1 = 0, hNrmInf = 0, cNrm1 = 0, cNrmInf = 0, ginf = 1, omega0 = 1;
  bool needs_single = false;  // resolving fallback: re-solved alone after the batch
  bool anchored = false;      // FP32 mode: deltas live (from the start of iterating to the halt)
  double t_done = 0;
  Req req;
  std::coroutine_handle<> waiting;
  Co<> task;
};

struct DevAwait {
  Inst* I;
  bool await_ready() const noexcept { return false; }
  void await_suspend(std::coroutine_handle<> h) noexcept { I->waiting = h; }
  void await_resume() const noexcept {}
};

static uint64_t fnv1a(const void* p, size_t n) {
  const unsigned char* b = static_cast<const unsigned char*>(p);
  uint64_t h = 1469598103934665603ull;
  for (size_t i = 0; i < n; ++i) {
    h ^= b[i];
    h *= 1099511628211ull;
  }
  return h;
}

// masked in-order copies / linear combinations (RQ_LIN)
struct LinList {
  LinOp op[6];
  int32_t count;
};

__global__ void masked_lin_kernel(LinList L, const int32_t* __restrict__ ix, const int32_t* __restrict__ iy,
                                  const uint8_t* __restrict__ mask, int64_t n, int64_t m) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int q = 0; q < L.count; ++q) {
    const LinOp& o = L.op[q];
    const int64_t len = o.side ? m : n;
    const int32_t* inst = o.side ? iy : ix;
    for (int64_t i = t0; i < len; i += stride) {
      if (!mask[inst[i]]) continue;
      o.dst[i] = o.a * o.u[i] + (o.v ? o.b * o.v[i] : 0.0);
    }
  }
}

// masked reflection (RQ_REFLECT): the host-side reflection after a checkpoint
__global__ void masked_reflect_kernel(const PdhgState* __restrict__ sts, const int32_t* __restrict__ ix,
                                      const int32_t* __restrict__ iy, const uint8_t* __restrict__ mask,
                                      double* __restrict__ x, double* __restrict__ xl, double* __restrict__ xm,
                                      int64_t n, double* __restrict__ y, double* __restrict__ yl,
                                      double* __restrict__ ym, int64_t m) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n + m; i += stride) {
    const bool isx = i < n;
    const int64_t j = isx ? i : i - n;
    const int32_t k = isx ? ix[j] : iy[j];
    if (!mask[k]) continue;
    const PdhgState& s = sts[k];
    double* v = isx ? x : y;
    double* vl = isx ? xl : yl;
    double* vm = isx ? xm : ym;
    const double tmp = s.refl_tmp, inv = s.refl_inv, e = s.refl_extra, eta = s.refl_eta, cum = s.refl_cum;
    const double cur = v[j];
    const double nv = tmp * ((1.0 + e) * cur - e * vl[j]) + inv * cur;
    vm[j] = (vm[j] * cum + nv * eta) / (cum + eta);
    v[j] = nv;
    vl[j] = nv;
  }
}

// ---------------------------------------------------------------------------
// The batched solver.
// ---------------------------------------------------------------------------
class BatchSolver : public Solver {
 public:
  BatchSolver(int64_t K, const pdcs_problem* probs, const pdcs_options* o)
      : Solver(probs, o), K_(K), probs_(probs) {}
  ~BatchSolver() override {
    for (int t = 0; t < 2; ++t) {
      if (bgraph_exec_[t]) cudaGraphExecDestroy(bgraph_exec_[t]);
      if (bgraph_[t]) cudaGraphDestroy(bgraph_[t]);
      for (cudaEvent_t e : gev_[t])
        if (e) cudaEventDestroy(e);
      if (round_ev_[t]) cudaEventDestroy(round_ev_[t]);
    }
    if (pin_) cudaFreeHost(pin_);
  }
  // merge, upload and precondition once (the problems must stay valid until destruction:
  // the resolving fallback re-solves an instance from them)
  int prepare();
  // cold-start solve of the prepared batch; attempt_limit > 0 overrides the option
  int solve(pdcs_result* res, pdcs_batch_info* info, int64_t attempt_limit);
  int run_batch(pdcs_result* res, pdcs_batch_info* info) {
    int rc = prepare();
    return rc != PDCS_OK ? rc : solve(res, info, 0);
  }
  // Solution-map adjoint at the last solve's solution (differentiable mode):
  // per-instance loss gradients dL/dx*, dL/dy* in, parameter gradients out
  // (any array may be NULL).  Arrays are indexed by instance.
  int grad(const double* const* dldx, const double* const* dldy, double* const* dc, double* const* dh,
           double* const* dG, double* const* dl, double* const* du, const pdcs_grad_options& go,
           pdcs_grad_info* info);
  // set the solution the adjoint differentiates at (instance-local host arrays)
  void set_solution(const double* const* xs, const double* const* ys);

 private:
  struct InstConst {
    double hNrm1, hNrmInf, cNrm1, cNrmInf, ginf, omega0;
  };
  std::vector<InstConst> consts_;
  double setup_time_ = 0.0;
  bool prepared_ = false;
  void reset_state();
  int64_t K_;
  const pdcs_problem* probs_;
  // merged host problem
  std::vector<int32_t> h_rp_;
  std::vector<int64_t> h_src_, nnz_off_;  // per merged row: its first nonzero in the instance-concatenated arrays
  std::vector<double> h_c_, h_h_, h_bl_, h_bu_;
  int32_t dummy_ci_ = 0;  // the merged matrix is assembled on the device (upload_matrix);
  double dummy_v_ = 0.0;  // these only stand for its column / value arrays in the host checks
  void upload_matrix(int32_t* g_rp, int32_t* g_ci, double* g_v) override;
  std::vector<int64_t> h_socx_, h_rsocx_, h_socG_, h_rsocG_;
  // per instance: offsets of its runs in the merged vectors and local starts
  std::vector<int64_t> xrun_start_, xrun_len_, yrun_start_, yrun_len_;  // K * kMaxRuns
  std::vector<int64_t> xloc_, yloc_;                                    // K * kMaxRuns local starts
  std::vector<int32_t> h_ix_, h_iy_;
  // per instance and side (0 = x, 1 = y): its warp cones [soc_first, soc_end) and
  // [rsoc_first, rsoc_end) in the side's cone list, its exp cone ordinals
  // [exp_first, exp_end) and dual-exp ordinals [dexp_first, dexp_end)
  std::vector<std::array<int64_t, 8>> cones_[2];
  std::vector<int8_t> cone_cls_[2];  // size class of every warp cone
  // differentiable mode
  bool solved_ = false;
  double *xs_raw_ = nullptr, *ys_raw_ = nullptr;  // the solution in the original scale (merged)
  ConeTable XA_{}, YA_{};                         // unscaled cone tables of X and K_d*
  struct Adj {
    int mr = 0;
    double *V = nullptr, *g = nullptr, *u = nullptr, *Au = nullptr, *coef = nullptr;
    double *a = nullptr, *b = nullptr, *xp = nullptr, *tw = nullptr, *tsw = nullptr, *tt = nullptr, *tq = nullptr,
           *tr = nullptr, *ttr = nullptr, *ts = nullptr, *dG = nullptr, *Tx = nullptr, *Sy = nullptr;
    double *dots1 = nullptr, *dots2 = nullptr, *dotsn = nullptr;
    double* dpart = nullptr;  // partial dot products: K x kAdjSplit x 8
    uint8_t* mask = nullptr;
    // GMRES state per instance on the device: Hessenberg matrix, rotations, rotated
    // right-hand side, initial residual norm, residual estimate, basis size, steps
    double *H = nullptr, *cs = nullptr, *sn = nullptr, *gam = nullptr, *beta0 = nullptr, *res = nullptr;
    int32_t* jk = nullptr;
    int64_t* iters = nullptr;
    uint8_t* run = nullptr;
  } adj_;
  static constexpr int kAdjSplit = 16;  // at most this many CTAs per instance in the adjoint's dot products
  void setup_adjoint(int mr);
  void apply_AT(const double* u, double* out, const uint8_t* mask);
  void scatter_x(const double* merged, double* const* out) const;
  void scatter_y(const double* merged, double* const* out) const;
  int64_t merged_row(int64_t k, int64_t i) const {
    int t = kMaxRuns - 1;
    while (t > 0 && i < yloc_[k * kMaxRuns + t]) --t;
    return yrun_start_[k * kMaxRuns + t] + (i - yloc_[k * kMaxRuns + t]);
  }
  // device
  int32_t *ix_ = nullptr, *iy_ = nullptr;
  RunTable rx_{}, ry_{};
  PdhgState* sts_ = nullptr;
  double *ps_ = nullptr, *ds_ = nullptr;
  uint8_t* live_ = nullptr;
  int32_t* live_cnt_ = nullptr;  // [0..1] live counts of alternating attempts, [2] accumulator
  uint32_t* done_ctas_ = nullptr;
  uint8_t* mask_ = nullptr;
  double *s0_ = nullptr, *s1_ = nullptr;
  double *cx_ = nullptr, *cy_ = nullptr;  // contributions: 8 x n, 8 x m
  double *dxsq_ = nullptr, *dysq_ = nullptr, *dgdy_ = nullptr;
  double* seg_out_ = nullptr;  // K * 20
  int64_t* cones_dev_[2] = {};  // cones_ on the device
  double* bs_prm_ = nullptr;    // K * 4
  double* bs_out_ = nullptr;    // K * 5
  int32_t* bs_list_ = nullptr;  // K
  // instance-tiled SpMVs of the iteration graph: [0] G (rows y, columns x), [1] G'
  struct Tiles {
    TileCsr T{};
    std::vector<int64_t> first;  // K + 1: tile range of every instance
    std::vector<int64_t> nnz;    // nonzeros of every tile
    int grid = 1;
  } tl_[2];
  bool tiled_ = false;
  // a tile holds up to kTileNnz nonzeros (spmv_tiles > 0 sets it): small enough that
  // the largest tiles do not leave SMs idle at the end, large enough that staging the
  // instance's columns (from L2) stays a fraction of the stream; tiles of instances
  // with few columns may hold up to 16 x their columns
  static constexpr int64_t kTileNnz = 65536;
  static constexpr int64_t kTileSmallNnz = 8192;
  static constexpr int64_t kTileMaxRows = 4096;
  static constexpr size_t kTileMaxSmem = 160 * 1024;
  void setup_tiles();
  // fused tile kernels of the full iteration graph (SELL-32 rows, the step and
  // projections of the tile's rows, per-tile partial sums): [0] G, the dual
  // step of y's rows; [1] G', the primal step of x's rows.  Used when the
  // batch has instance tiles and every SOC / RSOC block has at most 32 elements.
  struct Fused {
    FusedCsr F{};
    std::vector<int64_t> first;    // K + 1: tile range of every instance
    std::vector<int64_t> nnz;      // nonzeros of every tile
    int64_t* first_dev = nullptr;  // the same on the device (control sums)
    double* tpart = nullptr;       // per-tile partial sums (1 for G', 2 for G)
    float* sv32 = nullptr;         // SELL values: FP32 bulk ...
    double* sv64 = nullptr;        // ... or FP64
    int grid = 1;
  } fu_[2];
  bool fused_ = false;
  static constexpr int64_t kFusedMaxRows = 2048;
  void setup_fused();
  template <class T, int NV, class Op>
  int fused_grid(const FusedCsr& F, bool exp);
  // iteration graphs: [0] grids for the whole batch, [1] the tail graph, grids
  // capped for rounds in which few nonzeros iterate (most CTAs of the full
  // grids would find no work and return, at the cost of their launch)
  cudaGraph_t bgraph_[2] = {};
  cudaGraphExec_t bgraph_exec_[2] = {};
  static constexpr int kTailBinCtas = 64;     // SpMV CTAs per row bin
  // verbose timing: device time of each round (round_ev_), and with verbose >= 2
  // event nodes around the 6 kernels of every graph's last attempt (gev_)
  cudaEvent_t round_ev_[2] = {};
  cudaEvent_t gev_[2][7] = {};
  double gev_ms_[2][6] = {};
  int64_t gev_n_[2] = {};
  double dev_ms_ = 0.0;
  static constexpr int kTailCtas = 148;       // CTAs per part of the other kernels
  // the tail graph runs while fewer than kTailNnz nonzeros, and 1/16 of the batch's, iterate
  static constexpr int64_t kTailNnz = 1 << 20;
  // ... and when none of the iterating instances has more than kTailCtaNnz nonzeros,
  // tail_attempts_kernel runs them instead, a CTA per instance looping over its attempts
  static constexpr int64_t kTailCtaNnz = 32768;
  // active-row lists of G (0) and G' (1) for the iteration graph
  struct Compact {
    int4* rows = nullptr;
    int64_t* cbin = nullptr;
    int64_t* full_bin = nullptr;
    int32_t* flag = nullptr;
    int32_t* pos = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
  } cmp_[2];
  CsrDev Gc_{}, Gtc_{};
  CsrT<float> G32c_{}, Gt32c_{};
  void setup_compaction();
  void compact(const uint8_t* mask);
  // pinned staging (reset at every synchronisation)
  char* pin_ = nullptr;
  size_t pin_cap_ = 0, pin_off_ = 0;
  std::vector<Inst> inst_;
  int64_t rounds_ = 0;
  int64_t tail_rounds_ = 0;  // iteration rounds run by tail_attempts_kernel
  // host wall time per service request type (verbose report)
  double svc_s_[16] = {};
  int64_t svc_groups_[16] = {}, svc_insts_[16] = {};
  double iter_s_ = 0.0;

  int validate_batch();
  void merge();
  void setup_batch();
  // active work lists of the iteration graph (rebuilt when the iterating set changes)
  struct ActDev {
    int2* chunk = nullptr;
    int64_t* meta = nullptr;
    int64_t* sched = nullptr;
    int4* desc = nullptr;  // the scheduled cones' records (ConeTable::act_desc)
    int32_t* exp = nullptr;
  } act_[2];
  std::vector<int4> cone_desc_[2];  // per warp cone: {start, length | RSOC << 30, cone, instance}
  int4* rchunk_ = nullptr;
  int64_t* n_rchunk_ = nullptr;
  int32_t* act_inst_ = nullptr;
  int64_t* n_act_ = nullptr;
  ConeTable XIg_{}, YIg_{};  // XI / YI reading the active lists
  std::vector<uint8_t> act_set_;  // iterating set the lists describe
  size_t act_bytes_ = 0;          // largest upload of the lists
  void setup_act_lists();
  void build_act_lists(const std::vector<Inst*>& its);
  void capture_batch_graph(int tail);
  template <class T>
  T* stage(size_t count);
  void sync_reset() {
    PDCS_CUDA(cudaStreamSynchronize(s_));
    pin_off_ = 0;
  }
  uint8_t* upload_mask(const std::vector<Inst*>& g);
  void seg_launch(const uint8_t* mask, const SegSide& X, const SegSide& Y, int stride);
  const double* seg_fetch(int stride);
  void exec_group(std::vector<Inst*>& g);
  void exec_iterate(std::vector<Inst*>& its);
  void resume(Inst& I) {
    auto h = I.waiting;
    I.waiting = nullptr;
    h.resume();
    I.task.rethrow();
  }
  void schedule();

  // ---- requests (set the payload, suspend) ----
  DevAwait post(Inst& I, const ReqPayload& p, double s0 = 0.0, double s1 = 0.0, double s2 = 0.0, double s3 = 0.0) {
    I.req.key = p;
    I.req.hash = fnv1a(&I.req.key, sizeof(ReqPayload));
    I.req.s0 = s0;
    I.req.s1 = s1;
    I.req.s2 = s2;
    I.req.s3 = s3;
    return DevAwait{&I};
  }
  static ReqPayload payload(int32_t type) {
    ReqPayload p;
    std::memset(&p, 0, sizeof(p));  // padding takes part in the comparison
    p.type = type;
    return p;
  }
  struct Lin {
    double* dst;
    double a;
    const double* u;
    double b;
    const double* v;
    int side;
  };
  Co<> lin(Inst& I, std::vector<Lin> ops);
  Co<> converge_info(Inst& I, const double* xs, const double* ys, Converge& C, double* gxs, double* atys);
  Co<> exit_check(Inst& I);
  Co<double> mnorm(Inst& I, const double* dx, const double* dy, double ta, double si);
  Co<double> binary_search(Inst& I, double r, const double* px, const double* py, double ta, double si);
  Co<bool> binary_search_dev(Inst& I, double r, const double* px0, const double* py0, const double* px1,
                             const double* py1, double* vals);
  Co<double> approx(Inst& I, const ReqPayload& pr, double ta, double si, double& h1dx, double& h2dy, double t);
  Co<> restart_threshold(Inst& I, bool dgap);
  Co<bool> restart_check(Inst& I, bool dgap);
  Co<> omega_update(Inst& I, const double* xds, const double* yds);
  Co<> iterate(Inst& I);
  Co<> main_task(Inst& I);
  double kkt_error_i(const Inst& I, const Converge& C) const {
    const double om = I.S.omega;
    return std::sqrt(om * om * C.l2_abs_p * C.l2_abs_p + C.l2_abs_d * C.l2_abs_d / (om * om) +
                     C.abs_gap * C.abs_gap);
  }
};

template <class T>
T* BatchSolver::stage(size_t count) {
  size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
  if (pin_off_ + bytes > pin_cap_) sync_reset();
  if (bytes > pin_cap_) throw std::runtime_error("batch staging buffer too small");
  T* p = reinterpret_cast<T*>(pin_ + pin_off_);
  pin_off_ += bytes;
  return p;
}

int BatchSolver::validate_batch() {
  if (K_ < 1 || !probs_) return PDCS_ERR_INVALID;
  for (int64_t k = 0; k < K_; ++k) {
    const pdcs_problem& q = probs_[k];
    if (q.on_device) return PDCS_ERR_UNSUPPORTED;  // the batch merges host data
    Solver one(&q, &O);
    int rc = one.validate_only();
    if (rc != PDCS_OK) return rc;
    int64_t nsum = q.nb + 3 * (q.exp_x + q.dual_exp_x);
    for (int64_t i = 0; i < q.n_soc_x; ++i) nsum += q.soc_x[i];
    for (int64_t i = 0; i < q.n_rsoc_x; ++i) nsum += q.rsoc_x[i];
    if (nsum != q.n) return PDCS_ERR_N_MISMATCH;  // every variable belongs to a cone
    if (O.warm_start) return PDCS_ERR_UNSUPPORTED;
  }
  return PDCS_OK;
}

// Build the merged, type-ordered program on the host (parallel over instances).
void BatchSolver::merge() {
  const int64_t K = K_;
  std::vector<std::array<int64_t, kMaxRuns>> xs(K), ys(K);  // sizes per type
  for (int64_t k = 0; k < K; ++k) {
    const pdcs_problem& q = probs_[k];
    int64_t soc = 0, rsoc = 0, socg = 0, rsocg = 0;
    for (int64_t i = 0; i < q.n_soc_x; ++i) soc += q.soc_x[i];
    for (int64_t i = 0; i < q.n_rsoc_x; ++i) rsoc += q.rsoc_x[i];
    for (int64_t i = 0; i < q.n_socG; ++i) socg += q.socG[i];
    for (int64_t i = 0; i < q.n_rsocG; ++i) rsocg += q.rsocG[i];
    xs[k] = {q.nb, soc, rsoc, 3 * q.exp_x, 3 * q.dual_exp_x, 0};
    ys[k] = {q.mGzero, q.mGnonnegative, socg, rsocg, 3 * q.expG, 3 * q.dual_expG};
  }
  // region offsets and per-instance offsets inside each region
  xrun_start_.assign(K * kMaxRuns, 0);
  xrun_len_.assign(K * kMaxRuns, 0);
  yrun_start_.assign(K * kMaxRuns, 0);
  yrun_len_.assign(K * kMaxRuns, 0);
  xloc_.assign(K * kMaxRuns, 0);
  yloc_.assign(K * kMaxRuns, 0);
  int64_t N = 0, M = 0;
  for (int t = 0; t < kMaxRuns; ++t) {
    for (int64_t k = 0; k < K; ++k) {
      xrun_start_[k * kMaxRuns + t] = N;
      xrun_len_[k * kMaxRuns + t] = xs[k][t];
      N += xs[k][t];
      yrun_start_[k * kMaxRuns + t] = M;
      yrun_len_[k * kMaxRuns + t] = ys[k][t];
      M += ys[k][t];
    }
  }
  for (int64_t k = 0; k < K; ++k) {
    int64_t a = 0, b = 0;
    for (int t = 0; t < kMaxRuns; ++t) {
      xloc_[k * kMaxRuns + t] = a;
      a += xs[k][t];
      yloc_[k * kMaxRuns + t] = b;
      b += ys[k][t];
    }
  }
  // row lengths in merged order, then the merged CSR
  std::vector<int64_t>& nnz_off = nnz_off_;
  nnz_off.assign(K + 1, 0);
  for (int64_t k = 0; k < K; ++k) {
    const pdcs_problem& q = probs_[k];
    if (q.m > 0 && q.G_rowptr[q.m] - q.G_rowptr[0] != q.nnz) throw std::invalid_argument("csr");
    nnz_off[k + 1] = nnz_off[k] + probs_[k].nnz;
  }
  if (N > INT32_MAX || M > INT32_MAX || nnz_off[K] > INT32_MAX) throw std::invalid_argument("batch too large");
  h_rp_.assign(M + 1, 0);
  h_src_.assign(M, 0);
  h_c_.resize(N);
  h_h_.resize(M);
  h_ix_.resize(N);
  h_iy_.resize(M);
  int64_t NB = 0;
  for (int64_t k = 0; k < K; ++k) NB += probs_[k].nb;
  h_bl_.resize(NB);
  h_bu_.resize(NB);
  auto posx = [&](int64_t k, int64_t j) {
    int t = kMaxRuns - 1;
    while (t > 0 && j < xloc_[k * kMaxRuns + t]) --t;
    return xrun_start_[k * kMaxRuns + t] + (j - xloc_[k * kMaxRuns + t]);
  };
  auto posy = [&](int64_t k, int64_t i) {
    int t = kMaxRuns - 1;
    while (t > 0 && i < yloc_[k * kMaxRuns + t]) --t;
    return yrun_start_[k * kMaxRuns + t] + (i - yloc_[k * kMaxRuns + t]);
  };
  const unsigned nth = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  auto parallel = [&](auto&& fn) {
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nth; ++t)
      th.emplace_back([&, t]() {
        for (int64_t k = t; k < K; k += nth) fn(k);
      });
    for (auto& x : th) x.join();
  };
  parallel([&](int64_t k) {
    const pdcs_problem& q = probs_[k];
    for (int64_t i = 0; i < q.m; ++i) {
      const int64_t r = posy(k, i);
      h_rp_[r + 1] = q.G_rowptr[i + 1] - q.G_rowptr[i];
      h_src_[r] = nnz_off[k] + (q.G_rowptr[i] - q.G_rowptr[0]);
    }
    for (int64_t j = 0; j < q.n; ++j) {
      const int64_t p = posx(k, j);
      h_c_[p] = q.c[j];
      h_ix_[p] = (int32_t)k;
    }
    for (int64_t i = 0; i < q.m; ++i) {
      const int64_t p = posy(k, i);
      h_h_[p] = q.h[i];
      h_iy_[p] = (int32_t)k;
    }
    for (int64_t j = 0; j < q.nb; ++j) {
      h_bl_[xrun_start_[k * kMaxRuns] + j] = q.bl[j];
      h_bu_[xrun_start_[k * kMaxRuns] + j] = q.bu[j];
    }
  });
  for (int64_t i = 0; i < M; ++i) h_rp_[i + 1] += h_rp_[i];
  for (int w = 0; w < 2; ++w) cones_[w].assign(K, {});
  for (int64_t k = 0; k < K; ++k) {
    const pdcs_problem& q = probs_[k];
    cones_[0][k][0] = (int64_t)h_socx_.size();
    cones_[1][k][0] = (int64_t)h_socG_.size();
    h_socx_.insert(h_socx_.end(), q.soc_x, q.soc_x + q.n_soc_x);
    h_socG_.insert(h_socG_.end(), q.socG, q.socG + q.n_socG);
    cones_[0][k][1] = (int64_t)h_socx_.size();
    cones_[1][k][1] = (int64_t)h_socG_.size();
  }
  for (int64_t k = 0; k < K; ++k) {
    const pdcs_problem& q = probs_[k];
    cones_[0][k][2] = (int64_t)(h_socx_.size() + h_rsocx_.size());
    cones_[1][k][2] = (int64_t)(h_socG_.size() + h_rsocG_.size());
    h_rsocx_.insert(h_rsocx_.end(), q.rsoc_x, q.rsoc_x + q.n_rsoc_x);
    h_rsocG_.insert(h_rsocG_.end(), q.rsocG, q.rsocG + q.n_rsocG);
    cones_[0][k][3] = (int64_t)(h_socx_.size() + h_rsocx_.size());
    cones_[1][k][3] = (int64_t)(h_socG_.size() + h_rsocG_.size());
  }
  {
    int64_t ex = 0, ey = 0, dx = 0, dy = 0, EX = 0, EY = 0;
    for (int64_t k = 0; k < K; ++k) {
      EX += probs_[k].exp_x;
      EY += probs_[k].expG;
    }
    for (int64_t k = 0; k < K; ++k) {
      const pdcs_problem& q = probs_[k];
      cones_[0][k][4] = ex;
      cones_[0][k][5] = ex += q.exp_x;
      cones_[0][k][6] = EX + dx;
      cones_[0][k][7] = EX + (dx += q.dual_exp_x);
      cones_[1][k][4] = ey;
      cones_[1][k][5] = ey += q.expG;
      cones_[1][k][6] = EY + dy;
      cones_[1][k][7] = EY + (dy += q.dual_expG);
    }
  }
  for (int w = 0; w < 2; ++w) {
    const std::vector<int64_t>& soc = w ? h_socG_ : h_socx_;
    const std::vector<int64_t>& rsoc = w ? h_rsocG_ : h_rsocx_;
    cone_cls_[w].clear();
    for (const std::vector<int64_t>* L : {&soc, &rsoc})
      for (int64_t d : *L) {
        int c = 0;
        while (c < kCls - 1 && d > (2 << c)) ++c;  // the classes of the cone tables' schedule
        cone_cls_[w].push_back((int8_t)c);
      }
  }
  pdcs_problem mp;
  std::memset(&mp, 0, sizeof(mp));
  mp.n = N;
  mp.m = M;
  mp.nb = NB;
  mp.nnz = nnz_off[K];
  mp.G_rowptr = h_rp_.data();
  mp.G_colind = &dummy_ci_;
  mp.G_val = &dummy_v_;
  mp.c = h_c_.data();
  mp.h = h_h_.data();
  mp.bl = h_bl_.data();
  mp.bu = h_bu_.data();
  for (int64_t k = 0; k < K; ++k) {
    mp.mGzero += probs_[k].mGzero;
    mp.mGnonnegative += probs_[k].mGnonnegative;
    mp.expG += probs_[k].expG;
    mp.dual_expG += probs_[k].dual_expG;
    mp.exp_x += probs_[k].exp_x;
    mp.dual_exp_x += probs_[k].dual_exp_x;
  }
  mp.socG = h_socG_.data();
  mp.n_socG = (int64_t)h_socG_.size();
  mp.rsocG = h_rsocG_.data();
  mp.n_rsocG = (int64_t)h_rsocG_.size();
  mp.soc_x = h_socx_.data();
  mp.n_soc_x = (int64_t)h_socx_.size();
  mp.rsoc_x = h_rsocx_.data();
  mp.n_rsoc_x = (int64_t)h_rsocx_.size();
  mp.on_device = 0;
  P = mp;
}

// Host -> device copy of many pageable host segments into one contiguous
// device range.  A copy from pageable memory is staged by the driver one
// buffer at a time; here host threads gather the segments into pinned chunks
// while the copy engine moves the chunks filled before them.  Every thread
// owns two pinned chunks of a per-device ring, kept for the life of the
// process (kStageThreads x 2 x kStageChunk bytes, allocated on the first
// batch upload of a device) and guarded by a mutex, so concurrent batch
// setups on one device take turns.  The copies run on stream s; a chunk is
// refilled only after the event of its previous copy has completed.
struct HostSeg {
  const void* p;
  size_t bytes;
};
constexpr int kStageThreads = 8;
constexpr size_t kStageChunk = size_t(8) << 20;

class StageRing {
 public:
  static StageRing& of_current_device() {
    static std::mutex mu;
    static std::map<int, StageRing*> rings;
    int dev = 0;
    PDCS_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    StageRing*& r = rings[dev];
    if (!r) r = new StageRing();  // kept until exit: pinned buffers are process-wide
    return *r;
  }
  // Copies the concatenation of segs (total bytes) to dst.
  void upload(void* dst, const std::vector<HostSeg>& segs, cudaStream_t s) {
    std::lock_guard<std::mutex> lock(mu_);
    std::vector<size_t> pre(segs.size() + 1, 0);
    for (size_t i = 0; i < segs.size(); ++i) pre[i + 1] = pre[i] + segs[i].bytes;
    const size_t total = pre.back();
    if (total == 0) return;
    const size_t nchunks = (total + kStageChunk - 1) / kStageChunk;
    const int nth = (int)std::min<size_t>(kStageThreads, nchunks);
    if (!buf_[0]) {
      for (int i = 0; i < 2 * kStageThreads; ++i) {
        PDCS_CUDA(cudaHostAlloc(&buf_[i], kStageChunk, cudaHostAllocPortable));
        PDCS_CUDA(cudaEventCreateWithFlags(&ev_[i], cudaEventDisableTiming));
        PDCS_CUDA(cudaEventRecord(ev_[i], s));
      }
    }
    int dev = 0;
    PDCS_CUDA(cudaGetDevice(&dev));
    std::exception_ptr err = nullptr;
    std::mutex emu;
    auto work = [&](int t) {
      try {
        PDCS_CUDA(cudaSetDevice(dev));
        for (size_t c = (size_t)t, it = 0; c < nchunks; c += (size_t)nth, ++it) {
          const int slot = 2 * t + (int)(it & 1);
          PDCS_CUDA(cudaEventSynchronize(ev_[slot]));  // its previous copy has left the chunk
          const size_t a = c * kStageChunk, b = std::min(total, a + kStageChunk);
          size_t i = (size_t)(std::upper_bound(pre.begin(), pre.end(), a) - pre.begin()) - 1;
          unsigned char* out = static_cast<unsigned char*>(buf_[slot]);
          for (size_t pos = a; pos < b; ++i) {
            const size_t s0 = pos - pre[i], len = std::min(b, pre[i + 1]) - pos;
            if (len) std::memcpy(out + (pos - a), static_cast<const unsigned char*>(segs[i].p) + s0, len);
            pos += len;
          }
          PDCS_CUDA(cudaMemcpyAsync(static_cast<unsigned char*>(dst) + a, out, b - a, cudaMemcpyHostToDevice, s));
          PDCS_CUDA(cudaEventRecord(ev_[slot], s));
        }
      } catch (...) {
        std::lock_guard<std::mutex> lk(emu);
        err = std::current_exception();
      }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nth; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& x : th) x.join();
    if (err) std::rethrow_exception(err);
  }

 private:
  std::mutex mu_;
  void* buf_[2 * kStageThreads] = {};
  cudaEvent_t ev_[2 * kStageThreads] = {};
};

// The merged CSR of G, assembled on the device: every instance's column
// indices and values are uploaded as they are (concatenated in instance
// order, through the pinned staging ring), then merge_cols_kernel moves each
// merged row's nonzeros into place with the columns mapped to their merged
// positions (and checked against the instance's column count).
void BatchSolver::upload_matrix(int32_t* g_rp, int32_t* g_ci, double* g_v) {
  const int64_t K = K_;
  PDCS_CUDA(cudaMemcpyAsync(g_rp, h_rp_.data(), sizeof(int32_t) * (m_ + 1), cudaMemcpyHostToDevice, s_));
  if (nnz_ == 0) return;
  int32_t* ci_in = A.alloc<int32_t>(nnz_);
  double* v_in = A.alloc<double>(nnz_);
  {
    std::vector<HostSeg> sci, sv;
    sci.reserve(K);
    sv.reserve(K);
    for (int64_t k = 0; k < K; ++k) {
      const pdcs_problem& q = probs_[k];
      if (!q.nnz) continue;
      const int64_t o = q.G_rowptr[0];
      sci.push_back({q.G_colind + o, sizeof(int32_t) * (size_t)q.nnz});
      sv.push_back({q.G_val + o, sizeof(double) * (size_t)q.nnz});
    }
    StageRing& ring = StageRing::of_current_device();
    ring.upload(ci_in, sci, s_);  // nnz_off_ is the running sum of the instances' nnz in this order
    ring.upload(v_in, sv, s_);
  }
  std::vector<int64_t> ncol(K);
  for (int64_t k = 0; k < K; ++k) ncol[k] = probs_[k].n;
  int64_t* src = A.alloc<int64_t>(m_);
  int32_t* row_inst = A.alloc<int32_t>(m_);
  int64_t* xs = A.alloc<int64_t>(K * kMaxRuns);
  int64_t* xl = A.alloc<int64_t>(K * kMaxRuns);
  int64_t* nc = A.alloc<int64_t>(K);
  int32_t* err = A.alloc<int32_t>(1);
  PDCS_CUDA(cudaMemcpyAsync(src, h_src_.data(), sizeof(int64_t) * m_, cudaMemcpyHostToDevice, s_));
  PDCS_CUDA(cudaMemcpyAsync(row_inst, h_iy_.data(), sizeof(int32_t) * m_, cudaMemcpyHostToDevice, s_));
  PDCS_CUDA(cudaMemcpyAsync(xs, xrun_start_.data(), sizeof(int64_t) * K * kMaxRuns, cudaMemcpyHostToDevice, s_));
  PDCS_CUDA(cudaMemcpyAsync(xl, xloc_.data(), sizeof(int64_t) * K * kMaxRuns, cudaMemcpyHostToDevice, s_));
  PDCS_CUDA(cudaMemcpyAsync(nc, ncol.data(), sizeof(int64_t) * K, cudaMemcpyHostToDevice, s_));
  PDCS_CUDA(cudaMemsetAsync(err, 0, sizeof(int32_t), s_));
  merge_cols_kernel<<<warp_grid(m_), kThreads, 0, s_>>>(m_, g_rp, src, row_inst, ci_in, v_in, xs, xl, nc, g_ci, g_v, err);
  int32_t h_err = 0;
  PDCS_CUDA(cudaMemcpyAsync(&h_err, err, sizeof(int32_t), cudaMemcpyDeviceToHost, s_));
  PDCS_CUDA(cudaStreamSynchronize(s_));  // also keeps ncol alive for its copy
  for (const void* p : {(const void*)ci_in, (const void*)v_in, (const void*)src, (const void*)row_inst,
                        (const void*)xs, (const void*)xl, (const void*)nc, (const void*)err})
    A.drop(p);
  if (h_err) throw std::invalid_argument("csr");
}

void BatchSolver::setup_batch() {
  const int64_t K = K_;
  auto up = [&](auto* dst, const auto& v) {
    if (!v.empty()) PDCS_CUDA(cudaMemcpyAsync(dst, v.data(), v.size() * sizeof(v[0]), cudaMemcpyHostToDevice, s_));
  };
  ix_ = A.alloc<int32_t>(n_);
  iy_ = A.alloc<int32_t>(m_);
  up(ix_, h_ix_);
  up(iy_, h_iy_);
  int64_t* rxs = A.alloc<int64_t>(K * kMaxRuns);
  int64_t* rxl = A.alloc<int64_t>(K * kMaxRuns);
  int64_t* rys = A.alloc<int64_t>(K * kMaxRuns);
  int64_t* ryl = A.alloc<int64_t>(K * kMaxRuns);
  up(rxs, xrun_start_);
  up(rxl, xrun_len_);
  up(rys, yrun_start_);
  up(ryl, yrun_len_);
  rx_ = RunTable{rxs, rxl};
  ry_ = RunTable{rys, ryl};
  sts_ = A.alloc<PdhgState>(K);
  ps_ = A.alloc<double>(K);
  ds_ = A.alloc<double>(K);
  live_ = A.alloc<uint8_t>(K);
  live_cnt_ = A.alloc<int32_t>(4);
  done_ctas_ = A.alloc<uint32_t>(1);
  mask_ = A.alloc<uint8_t>(K);
  s0_ = A.alloc<double>(K);
  s1_ = A.alloc<double>(K);
  cx_ = A.alloc<double>(8 * std::max<int64_t>(n_, 1));
  cy_ = A.alloc<double>(8 * std::max<int64_t>(m_, 1));
  dxsq_ = A.alloc<double>(n_);
  dysq_ = A.alloc<double>(m_);
  dgdy_ = A.alloc<double>(m_);
  seg_out_ = A.alloc<double>(K * 20);
  bs_prm_ = A.alloc<double>(4 * K);
  bs_out_ = A.alloc<double>(5 * K);
  bs_list_ = A.alloc<int32_t>(K);
  for (int w = 0; w < 2; ++w) {
    cones_dev_[w] = A.alloc<int64_t>(8 * K);
    PDCS_CUDA(cudaMemcpyAsync(cones_dev_[w], cones_[w].data(), sizeof(int64_t) * 8 * K, cudaMemcpyHostToDevice, s_));
  }
  PDCS_CUDA(cudaMemsetAsync(live_cnt_, 0, 4 * sizeof(int32_t), s_));
  PDCS_CUDA(cudaMemsetAsync(done_ctas_, 0, sizeof(uint32_t), s_));
  PDCS_CUDA(cudaMemsetAsync(live_, 0, K, s_));
  pin_cap_ = std::max<size_t>(size_t(1) << 20, (size_t)K * (20 * sizeof(double) + sizeof(PdhgState)) * 4 + 4096);
  PDCS_CUDA(cudaMallocHost(&pin_, pin_cap_));
  consts_.resize(K);
  // per-instance constants: raw norms (cal_constant), ginf, initial primal weight
  {
    SegSide X{}, Y{};
    X.a[0] = c_raw; X.kind[0] = SK_SUMABS;
    X.a[1] = c_raw; X.kind[1] = SK_MAXABS;
    X.a[2] = c_s; X.kind[2] = SK_DOT;
    X.count = 3;
    double* rowmax = tm[0];
    row_absstat_kernel<false><<<warp_grid(m_), kThreads, 0, s_>>>(m_, G_.rp, G_.v, nullptr, rowmax);
    Y.a[0] = h_raw; Y.kind[0] = SK_SUMABS;
    Y.a[1] = h_raw; Y.kind[1] = SK_MAXABS;
    Y.a[2] = h_s; Y.kind[2] = SK_DOT;
    Y.a[3] = rowmax; Y.kind[3] = SK_MAX;
    Y.count = 4;
    seg_launch(nullptr, X, Y, 7);
    const double* r = seg_fetch(7);
    for (int64_t k = 0; k < K; ++k) {
      InstConst& I = consts_[k];
      const double* q = r + k * 7;
      I.cNrm1 = q[0];
      I.cNrmInf = q[1];
      I.hNrm1 = q[3];
      I.hNrmInf = q[4];
      I.ginf = q[6];
      const double cn = std::sqrt(q[2]), hn = std::sqrt(q[5]);
      I.omega0 = (hn > 1e-10 && cn > 1e-10) ? cn / hn : 1.0;
    }
  }
  attempts_per_graph_ = (attempts_per_graph_ + 1) & ~1;  // even: live-count slots alternate
}

uint8_t* BatchSolver::upload_mask(const std::vector<Inst*>& g) {
  uint8_t* h = stage<uint8_t>(K_);
  std::memset(h, 0, K_);
  for (Inst* I : g) h[I->k] = 1;
  PDCS_CUDA(cudaMemcpyAsync(mask_, h, K_, cudaMemcpyHostToDevice, s_));
  return mask_;
}

void BatchSolver::seg_launch(const uint8_t* mask, const SegSide& X, const SegSide& Y, int stride) {
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((K_ * 32 + kThreads - 1) / kThreads, 148 * 16));
  seg_reduce_kernel<<<grid, kThreads, 0, s_>>>(K_, mask, rx_, X, ry_, Y, seg_out_, stride);
  kernels_++;
}

const double* BatchSolver::seg_fetch(int stride) {
  double* h = stage<double>((size_t)K_ * stride);
  PDCS_CUDA(cudaMemcpyAsync(h, seg_out_, sizeof(double) * K_ * stride, cudaMemcpyDeviceToHost, s_));
  PDCS_CUDA(cudaStreamSynchronize(s_));
  // the staged copy stays valid until the next stage() call wraps around
  return h;
}

void BatchSolver::setup_compaction() {
  const CsrDev* full[2] = {&G_, &Gt_};
  CsrDev* view[2] = {&Gc_, &Gtc_};
  for (int w = 0; w < 2; ++w) {
    Compact& c = cmp_[w];
    const CsrDev& F = *full[w];
    const int64_t R = F.bin_off[kBins];
    c.rows = A.alloc<int4>(std::max<int64_t>(R, 1));
    c.cbin = A.alloc<int64_t>(kBins + 1);
    c.full_bin = A.alloc<int64_t>(kBins + 1);
    c.flag = A.alloc<int32_t>(R + 1);
    c.pos = A.alloc<int32_t>(R + 1);
    PDCS_CUDA(cudaMemcpyAsync(c.full_bin, F.bin_off, sizeof(int64_t) * (kBins + 1), cudaMemcpyHostToDevice, s_));
    PDCS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, c.tmp_bytes, c.flag, c.pos, (int)(R + 1), s_));
    c.tmp = A.alloc<char>(std::max<size_t>(c.tmp_bytes, 1));
    *view[w] = F;
    view[w]->rows = c.rows;
    view[w]->dbin = c.cbin;
  }
  PDCS_CUDA(cudaStreamSynchronize(s_));  // the bin offsets were copied from the host structs
  if (fp32_) {
    G32c_ = G32_;
    G32c_.rows = cmp_[0].rows;
    G32c_.dbin = cmp_[0].cbin;
    Gt32c_ = Gt32_;
    Gt32c_.rows = cmp_[1].rows;
    Gt32c_.dbin = cmp_[1].cbin;
  }
}

// Tiles of the instances' rows for both matrices (instance-tiled SpMV), when every
// instance has at most kTileMaxCols columns in either matrix and its column
// segment fits the shared-memory budget; otherwise the graph keeps the binned SpMV.
void BatchSolver::setup_tiles() {
  tiled_ = false;
  if (O.spmv_tiles < 0) return;
  int64_t maxc[2] = {0, 0};  // G: the instance's x; G': its y
  for (int64_t k = 0; k < K_; ++k) {
    maxc[0] = std::max<int64_t>(maxc[0], probs_[k].n);
    maxc[1] = std::max<int64_t>(maxc[1], probs_[k].m);
  }
  if (maxc[0] > kTileMaxCols || maxc[1] > kTileMaxCols) return;
  const size_t eb = fp32_ ? sizeof(float) : sizeof(double);
  const size_t smem[2] = {2 * eb * (size_t)maxc[0], eb * (size_t)maxc[1]};  // G stages (x, x_lag) pairs
  if (smem[0] > kTileMaxSmem || smem[1] > kTileMaxSmem) return;
  auto up32 = [&](const std::vector<int64_t>& v) {
    std::vector<int32_t> h(v.begin(), v.end());
    int32_t* d = A.alloc<int32_t>(h.size());
    PDCS_CUDA(cudaMemcpyAsync(d, h.data(), sizeof(int32_t) * h.size(), cudaMemcpyHostToDevice, s_));
    PDCS_CUDA(cudaStreamSynchronize(s_));  // h is a temporary
    return d;
  };
  int32_t* xloc = up32(xloc_);
  int32_t* yloc = up32(yloc_);
  std::vector<int32_t> rpt(n_ + 1);
  PDCS_CUDA(cudaMemcpyAsync(rpt.data(), Gt_.rp, sizeof(int32_t) * (n_ + 1), cudaMemcpyDeviceToHost, s_));
  PDCS_CUDA(cudaStreamSynchronize(s_));
  int dev = 0, sms = 148;
  PDCS_CUDA(cudaGetDevice(&dev));
  PDCS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  for (int w = 0; w < 2; ++w) {
    Tiles& t = tl_[w];
    const CsrDev& F = w ? Gt_ : G_;
    const std::vector<int32_t>& rp = w ? rpt : h_rp_;
    const std::vector<int64_t>& rs = w ? xrun_start_ : yrun_start_;  // row side
    const std::vector<int64_t>& rl = w ? xrun_len_ : yrun_len_;
    const std::vector<int64_t>& cs = w ? yrun_start_ : xrun_start_;  // column side
    const int64_t R = w ? n_ : m_;
    uint16_t* cl = A.alloc<uint16_t>(std::max<int64_t>(nnz_, 1));
    RegionStarts reg{};
    for (int q = 0; q < kMaxRuns; ++q) reg.s[q] = cs[q];  // instance 0 opens every type region
    local_cols_kernel<<<grid_for(R), kThreads, 0, s_>>>(R, F.rp, F.ci, w ? ix_ : iy_, reg, w ? ry_.start : rx_.start,
                                                        w ? yloc : xloc, cl);
    std::vector<int4> tiles;
    t.first.assign(K_ + 1, 0);
    t.nnz.clear();
    for (int64_t k = 0; k < K_; ++k) {
      t.first[k] = (int64_t)tiles.size();
      const int64_t ncols = w ? probs_[k].m : probs_[k].n;
      const int64_t big = O.spmv_tiles > 0 ? (int64_t)O.spmv_tiles : kTileNnz;
      const int64_t cap = std::min(big, std::max(kTileSmallNnz, 16 * ncols));
      int64_t o = 0, ob = 0, acc = 0;
      const int64_t ln = fp32_ ? kTileLN<float> : kTileLN<double>;
      auto cut = [&](int64_t end) {
        const int64_t rows = end - ob;
        int g = 1;
        while (g < 32 && ln * g * rows < acc) g *= 2;  // about ln nonzeros per lane
        tiles.push_back(make_int4((int32_t)k, (int32_t)ob, (int32_t)end, g));
        t.nnz.push_back(acc);
        ob = end;
        acc = 0;
      };
      for (int q = 0; q < kMaxRuns; ++q)
        for (int64_t i = 0; i < rl[k * kMaxRuns + q]; ++i, ++o) {
          const int64_t row = rs[k * kMaxRuns + q] + i;
          acc += rp[row + 1] - rp[row];
          if (acc >= cap || o + 1 - ob >= kTileMaxRows) cut(o + 1);
        }
      if (o > ob) cut(o);
    }
    t.first[K_] = (int64_t)tiles.size();
    int4* dt = A.alloc<int4>(std::max<size_t>(tiles.size(), 1));
    PDCS_CUDA(cudaMemcpyAsync(dt, tiles.data(), sizeof(int4) * tiles.size(), cudaMemcpyHostToDevice, s_));
    PDCS_CUDA(cudaStreamSynchronize(s_));  // tiles is a temporary
    TileCsr& T = t.T;
    T.rp = F.rp;
    T.cl = cl;
    T.tiles = dt;
    T.ntiles = (int64_t)tiles.size();
    T.act = A.alloc<int32_t>(std::max<size_t>(tiles.size(), 1));
    T.n_act = A.alloc<int64_t>(1);
    T.rows = w ? rx_ : ry_;
    T.cols = w ? ry_ : rx_;
    T.rloc = w ? xloc : yloc;
    T.cloc = w ? yloc : xloc;
    T.max_cols = (int32_t)maxc[w];
    const int per_sm = (int)std::max<size_t>(1, std::min<size_t>(2048 / kTileThreads, (size_t)(228 * 1024) / (smem[w] + 1024)));
    t.grid = (int)std::max<int64_t>(1, std::min<int64_t>(T.ntiles, (int64_t)sms * per_sm));
  }
  if (fp32_) {
    tile_prepare<float, kPair>(tl_[0].T);
    tile_prepare<float, 1>(tl_[1].T);
  } else {
    tile_prepare<double, 2>(tl_[0].T);
    tile_prepare<double, 1>(tl_[1].T);
  }
  tiled_ = true;
}

// Fused tiles (fused_tile_kernel) for both matrices.  A tile is a range of one
// instance's rows in the instance's own order, cut only between cones: its
// elementwise rows come first, then whole SOC / RSOC blocks, exponential and
// dual-exponential triples.  Per tile: the SELL-32 slices of its rows (sorted
// by length), the lane-group tasks of its blocks by size class, its exp records.
void BatchSolver::setup_fused() {
  fused_ = false;
  if (!tiled_) return;
  for (int w = 0; w < 2; ++w)
    for (int8_t c : cone_cls_[w])
      if (c >= kCls - 1) return;  // a block of more than 32 elements: the unfused kernels
  std::vector<int32_t> rpt(n_ + 1);
  PDCS_CUDA(cudaMemcpyAsync(rpt.data(), Gt_.rp, sizeof(int32_t) * (n_ + 1), cudaMemcpyDeviceToHost, s_));
  PDCS_CUDA(cudaStreamSynchronize(s_));
  // the layout of one instance, with instance-local offsets (concatenated below)
  struct Part {
    std::vector<FusedTile> tiles;
    std::vector<int64_t> sb, nnz;
    std::vector<int32_t> sl, srow;
    std::vector<int16_t> so;
    std::vector<int4> task, crec, xrec;
    int64_t pad = 0;
    int32_t max_rows = 1;
  };
  for (int w = 0; w < 2; ++w) {
    // w = 0: G, rows are y's elements (side 1 of the cone lists); w = 1: G', rows are x's (side 0)
    const int cs = w == 0 ? 1 : 0;
    const ConeTable& CT = w == 0 ? YI : XI;
    const std::vector<int32_t>& rp = w == 0 ? h_rp_ : rpt;
    const std::vector<int64_t>& rs = w == 0 ? yrun_start_ : xrun_start_;
    const std::vector<int64_t>& rl = w == 0 ? yrun_len_ : xrun_len_;
    const std::vector<int64_t>& lc = w == 0 ? yloc_ : xloc_;
    const int nelem_runs = w == 0 ? 2 : 1;  // y: zero, nonneg; x: box
    auto build = [&](int64_t k, Part& P) {
      struct Atom {
        int64_t ord, j;                 // instance-local ordinal and merged index of the first element
        int32_t size, type, id, flags;  // type 0 elementwise, 1 SOC / RSOC block, 2 exp triple
      };
      const int64_t nk = w == 0 ? probs_[k].m : probs_[k].n;
      std::vector<int64_t> mrow(nk), rlen(nk);  // merged row and length of every instance row
      for (int q = 0; q < kMaxRuns; ++q)
        for (int64_t i = 0; i < rl[k * kMaxRuns + q]; ++i) {
          const int64_t o = lc[k * kMaxRuns + q] + i, r = rs[k * kMaxRuns + q] + i;
          mrow[o] = r;
          rlen[o] = rp[r + 1] - rp[r];
        }
      auto ord_of = [&](int64_t j) {
        for (int q = 0; q < kMaxRuns; ++q) {
          const int64_t a = rs[k * kMaxRuns + q], L = rl[k * kMaxRuns + q];
          if (j >= a && j < a + L) return lc[k * kMaxRuns + q] + (j - a);
        }
        throw std::logic_error("fused tiles: element outside its instance's runs");
      };
      std::vector<Atom> at;
      at.reserve(nk);
      for (int q = 0; q < nelem_runs; ++q)
        for (int64_t i = 0; i < rl[k * kMaxRuns + q]; ++i)
          at.push_back({lc[k * kMaxRuns + q] + i, rs[k * kMaxRuns + q] + i, 1, 0, 0, 0});
      const std::array<int64_t, 8>& c = cones_[cs][k];
      for (int part = 0; part < 2; ++part)
        for (int64_t i = c[2 * part]; i < c[2 * part + 1]; ++i) {
          const int4 d = cone_desc_[cs][i];
          at.push_back({ord_of(d.x), d.x, d.y & 0x3fffffff, 1, (int32_t)i, d.y});
        }
      for (int part = 0; part < 2; ++part)
        for (int64_t kk = c[4 + 2 * part]; kk < c[5 + 2 * part]; ++kk) {
          const int64_t j = kk < CT.exp_count ? CT.exp_base + 3 * kk : CT.dexp_base + 3 * (kk - CT.exp_count);
          at.push_back({ord_of(j), j, 3, 2, (int32_t)kk, 0});
        }
      std::stable_sort(at.begin(), at.end(), [](const Atom& a, const Atom& b) { return a.ord < b.ord; });
      const int64_t ncols = w == 0 ? probs_[k].n : probs_[k].m;
      const int64_t big = O.spmv_tiles > 0 ? (int64_t)O.spmv_tiles : kTileNnz;
      const int64_t cap = std::min(big, std::max(kTileSmallNnz, 16 * ncols));
      size_t a0 = 0;
      int64_t rows = 0, acc = 0;
      std::vector<int32_t> loc;
      std::vector<int4> recs[kCls];
      auto cut = [&](size_t a1) {  // atoms [a0, a1) form a tile
        FusedTile T{};
        T.inst = (int32_t)k;
        T.o0 = (int32_t)at[a0].ord;
        T.o1 = (int32_t)(at[a1 - 1].ord + at[a1 - 1].size);
        int32_t ew = 0;
        for (size_t a = a0; a < a1 && at[a].type == 0; ++a) ew++;
        T.ew = ew;
        const int32_t nr = T.o1 - T.o0;
        P.max_rows = std::max(P.max_rows, nr);
        // SELL-32 slices of the tile's rows, longest first
        loc.resize(nr);
        for (int32_t i = 0; i < nr; ++i) loc[i] = i;
        std::stable_sort(loc.begin(), loc.end(), [&](int32_t a, int32_t b) { return rlen[T.o0 + a] > rlen[T.o0 + b]; });
        T.s0 = (int32_t)P.sl.size();
        for (int32_t i = 0; i < nr; i += kSellC) {
          const int32_t L = (int32_t)rlen[T.o0 + loc[i]];
          P.sb.push_back(P.pad);
          P.sl.push_back(L);
          for (int l = 0; l < kSellC; ++l) {
            const bool ok = i + l < nr;
            P.so.push_back(ok ? (int16_t)loc[i + l] : (int16_t)-1);
            P.srow.push_back(ok ? (int32_t)mrow[T.o0 + loc[i + l]] : -1);
          }
          P.pad += (int64_t)L * kSellC;
        }
        T.s1 = (int32_t)P.sl.size();
        // lane-group tasks of the blocks, class by class
        for (auto& r : recs) r.clear();
        for (size_t a = a0; a < a1; ++a)
          if (at[a].type == 1)
            recs[cone_cls_[cs][at[a].id]].push_back(
                make_int4((int32_t)at[a].j, at[a].flags, at[a].id, (int32_t)(at[a].ord - T.o0)));
        T.t0 = (int32_t)P.task.size();
        for (int cls = 0; cls < kCls - 1; ++cls) {  // blocks of <= 2 << cls elements
          const int g = std::max(1, (2 << cls) / kFusedEPL), per = 32 / g;
          for (size_t r = 0; r < recs[cls].size(); r += per) {
            const int cnt = (int)std::min<size_t>(per, recs[cls].size() - r);
            P.task.push_back(make_int4((int32_t)P.crec.size(), cnt, g, 0));
            P.crec.insert(P.crec.end(), recs[cls].begin() + r, recs[cls].begin() + r + cnt);
          }
        }
        T.t1 = (int32_t)P.task.size();
        T.x0 = (int32_t)P.xrec.size();
        for (size_t a = a0; a < a1; ++a)
          if (at[a].type == 2) P.xrec.push_back(make_int4((int32_t)at[a].j, at[a].id, (int32_t)(at[a].ord - T.o0), 0));
        T.x1 = (int32_t)P.xrec.size();
        P.tiles.push_back(T);
        P.nnz.push_back(acc);
        a0 = a1;
        rows = 0;
        acc = 0;
      };
      for (size_t a = 0; a < at.size(); ++a) {
        if (rows > 0 && rows + at[a].size > kFusedMaxRows) cut(a);
        for (int32_t e = 0; e < at[a].size; ++e) acc += rlen[at[a].ord + e];
        rows += at[a].size;
        if (acc >= cap) cut(a + 1);
      }
      if (a0 < at.size()) cut(at.size());
    };
    // instances in parallel, then concatenated in instance order
    std::vector<Part> parts(K_);
    {
      const int nth = (int)std::max<int64_t>(
          1, std::min<int64_t>(K_ / 64, (int64_t)std::max(1u, std::thread::hardware_concurrency())));
      std::vector<std::thread> th;
      std::exception_ptr err = nullptr;
      std::mutex emu;
      for (int t = 0; t < nth; ++t)
        th.emplace_back([&, t] {
          try {
            for (int64_t k = t; k < K_; k += nth) build(k, parts[k]);
          } catch (...) {
            std::lock_guard<std::mutex> lk(emu);
            err = std::current_exception();
          }
        });
      for (auto& x : th) x.join();
      if (err) std::rethrow_exception(err);
    }
    Fused& fu = fu_[w];
    Part all;
    fu.first.assign(K_ + 1, 0);
    for (int64_t k = 0; k < K_; ++k) {
      Part& P = parts[k];
      fu.first[k] = (int64_t)all.tiles.size();
      const int32_t so0 = (int32_t)all.sl.size(), to0 = (int32_t)all.task.size(), xo0 = (int32_t)all.xrec.size();
      const int32_t co0 = (int32_t)all.crec.size();
      for (FusedTile T : P.tiles) {
        T.s0 += so0;
        T.s1 += so0;
        T.t0 += to0;
        T.t1 += to0;
        T.x0 += xo0;
        T.x1 += xo0;
        all.tiles.push_back(T);
      }
      for (int64_t b : P.sb) all.sb.push_back(b + all.pad);
      for (int4 t : P.task) all.task.push_back(make_int4(t.x + co0, t.y, t.z, t.w));
      all.sl.insert(all.sl.end(), P.sl.begin(), P.sl.end());
      all.so.insert(all.so.end(), P.so.begin(), P.so.end());
      all.srow.insert(all.srow.end(), P.srow.begin(), P.srow.end());
      all.crec.insert(all.crec.end(), P.crec.begin(), P.crec.end());
      all.xrec.insert(all.xrec.end(), P.xrec.begin(), P.xrec.end());
      all.nnz.insert(all.nnz.end(), P.nnz.begin(), P.nnz.end());
      all.pad += P.pad;
      all.max_rows = std::max(all.max_rows, P.max_rows);
      P = Part();  // release as we go
    }
    fu.first[K_] = (int64_t)all.tiles.size();
    fu.nnz = std::move(all.nnz);
    std::vector<FusedTile>& tiles = all.tiles;
    std::vector<int64_t>& sb = all.sb;
    std::vector<int32_t>& sl = all.sl;
    std::vector<int16_t>& so = all.so;
    std::vector<int32_t>& srow = all.srow;
    std::vector<int4>& task = all.task;
    std::vector<int4>& crec = all.crec;
    std::vector<int4>& xrec = all.xrec;
    const int64_t pad = all.pad;
    const int32_t max_rows = all.max_rows;
    if (tiles.size() > (size_t)INT32_MAX || sl.size() > (size_t)INT32_MAX) return;
    {  // the layout's invariants, checked once on the host before any kernel reads it
      auto bad = [](const char* what) { throw std::logic_error(std::string("fused tiles: ") + what); };
      for (int64_t k = 0; k < K_; ++k) {
        const int64_t nk = w == 0 ? probs_[k].m : probs_[k].n;
        int64_t o = 0;
        for (int64_t t = fu.first[k]; t < fu.first[k + 1]; ++t) {
          const FusedTile& T = tiles[t];
          if (T.inst != k || T.o0 != o || T.o1 <= T.o0 || T.o1 - T.o0 > max_rows || T.ew > T.o1 - T.o0) bad("row ranges");
          o = T.o1;
          const int32_t nr = T.o1 - T.o0;
          std::vector<uint8_t> seen(nr, 0);
          for (int32_t sI = T.s0; sI < T.s1; ++sI)
            for (int l = 0; l < kSellC; ++l) {
              const int16_t v = so[(size_t)sI * kSellC + l];
              if (v < -1 || v >= nr || (v >= 0 && seen[v]++)) bad("slice slots");
            }
          for (int32_t i = 0; i < nr; ++i)
            if (!seen[i]) bad("a row without a slot");
          for (int32_t q = T.t0; q < T.t1; ++q)
            for (int r = 0; r < task[q].y; ++r) {
              const int4 cr = crec[task[q].x + r];
              if (cr.w < T.ew || cr.w + (cr.y & 0x3fffffff) > nr || (cr.y & 0x3fffffff) > task[q].z * kFusedEPL ||
                  (cr.y & 0x3fffffff) < (((cr.y >> 30) & 1) ? 3 : 2))
                bad("cone records");
            }
          for (int32_t q = T.x0; q < T.x1; ++q)
            if (xrec[q].z < T.ew || xrec[q].z + 3 > nr) bad("exp records");
        }
        if (o != nk) bad("rows of an instance not covered");
      }
    }
    // device copies
    auto up = [&](const auto& v) {
      using E = typename std::decay_t<decltype(v)>::value_type;
      E* d = A.alloc<E>(std::max<size_t>(v.size(), 1));
      if (!v.empty()) PDCS_CUDA(cudaMemcpyAsync(d, v.data(), sizeof(E) * v.size(), cudaMemcpyHostToDevice, s_));
      return d;
    };
    FusedCsr& F = fu.F;
    F.tiles = up(tiles);
    F.ntiles = (int64_t)tiles.size();
    F.act = A.alloc<int32_t>(std::max<size_t>(tiles.size(), 1));
    F.n_act = A.alloc<int64_t>(1);
    F.sb = up(sb);
    F.sl = up(sl);
    F.so = up(so);
    F.task = up(task);
    F.crec = up(crec);
    F.xrec = up(xrec);
    F.rows = w == 0 ? ry_ : rx_;
    F.cols = w == 0 ? rx_ : ry_;
    F.rloc = tl_[w].T.rloc;
    F.cloc = tl_[w].T.cloc;
    F.max_cols = tl_[w].T.max_cols;
    F.max_rows = max_rows;
    F.sched = A.alloc<int32_t>(2);
    PDCS_CUDA(cudaMemsetAsync(F.sched, 0, 2 * sizeof(int32_t), s_));
    fu.first_dev = up(fu.first);
    fu.tpart = A.alloc<double>(std::max<size_t>(tiles.size(), 1) * (w == 0 ? 2 : 1));
    int32_t* d_srow = up(srow);
    uint16_t* sc = A.alloc<uint16_t>(std::max<int64_t>(pad, 1));
    F.sc = sc;
    const int64_t nsl = (int64_t)sl.size();
    const int fg = (int)std::max<int64_t>(1, std::min<int64_t>((nsl * kSellC + kThreads - 1) / kThreads, 148 * 32));
    const CsrDev& M = w == 0 ? G_ : Gt_;
    if (fp32_) {
      fu.sv32 = A.alloc<float>(std::max<int64_t>(pad, 1));
      const CsrT<float>& M32 = w == 0 ? G32_ : Gt32_;
      sell_fill_kernel<float><<<fg, kThreads, 0, s_>>>(nsl, F.sb, F.sl, d_srow, M.rp, M32.v, tl_[w].T.cl, fu.sv32, sc);
    } else {
      fu.sv64 = A.alloc<double>(std::max<int64_t>(pad, 1));
      sell_fill_kernel<double><<<fg, kThreads, 0, s_>>>(nsl, F.sb, F.sl, d_srow, M.rp, M.v, tl_[w].T.cl, fu.sv64, sc);
    }
    PDCS_CUDA(cudaGetLastError());
    PDCS_CUDA(cudaStreamSynchronize(s_));  // the host vectors above are temporaries
  }
  const bool ex = XI.exp_count + XI.dexp_count > 0, ey = YI.exp_count + YI.dexp_count > 0;
  if (fp32_) {
    fu_[1].grid = fused_grid<float, 1, FusedPrimal32>(fu_[1].F, ex);
    fu_[0].grid = fused_grid<float, kPair, FusedDual32>(fu_[0].F, ey);
  } else {
    fu_[1].grid = fused_grid<double, 1, FusedPrimal64>(fu_[1].F, ex);
    fu_[0].grid = fused_grid<double, 2, FusedDual64>(fu_[0].F, ey);
  }
  fused_ = fu_[0].grid > 0 && fu_[1].grid > 0;
  if (O.verbose)
    std::printf("[pdcs_b200 setup] fused tiles: G %lld tiles, grid %d; G' %lld tiles, grid %d%s\n",
                (long long)fu_[0].F.ntiles, fu_[0].grid, (long long)fu_[1].F.ntiles, fu_[1].grid,
                fused_ ? "" : " (not used: shared memory)");
}

// CTAs of a fused kernel: resident CTAs per SM (registers and shared memory) x SMs,
// at most one per tile; 0 when one CTA does not fit.
template <class T, int NV, class Op>
int BatchSolver::fused_grid(const FusedCsr& F, bool exp) {
  const size_t smem = fused_smem_bytes<T, NV>(F);
  if (smem > 220 * 1024) return 0;
  int dev = 0, sms = 148, per = 0;
  PDCS_CUDA(cudaGetDevice(&dev));
  PDCS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (exp) {
    fused_prepare<T, NV, Op, true>(F);
    PDCS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fused_tile_kernel<T, NV, Op, true>, kFusedThreads, smem));
  } else {
    fused_prepare<T, NV, Op, false>(F);
    PDCS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fused_tile_kernel<T, NV, Op, false>, kFusedThreads, smem));
  }
  if (per <= 0) return 0;
  return (int)std::max<int64_t>(1, std::min<int64_t>(F.ntiles, (int64_t)sms * per));
}

// Device buffers of the active work lists, sized for every instance iterating.
void BatchSolver::setup_act_lists() {
  auto nchunks = [](int64_t len) { return (len + kThreads - 1) / kThreads; };
  const ConeTable* T[2] = {&XI, &YI};
  size_t bytes = 0;
  int64_t nr = 0;
  for (int w = 0; w < 2; ++w) {
    const std::vector<int64_t>& rl = w ? yrun_len_ : xrun_len_;
    int64_t nc = 0;
    for (int64_t k = 0; k < K_; ++k) {
      for (int q = 0; q < (w ? 2 : 1); ++q) nc += nchunks(rl[k * kMaxRuns + q]);
      for (int q = 0; q < kMaxRuns; ++q) nr += nchunks(rl[k * kMaxRuns + q]);
    }
    const int64_t ne = T[w]->exp_count + T[w]->dexp_count;
    act_[w].chunk = A.alloc<int2>(std::max<int64_t>(nc, 1));
    act_[w].meta = A.alloc<int64_t>(2 * kCls + 4);
    act_[w].sched = A.alloc<int64_t>(std::max<int64_t>(T[w]->nwc, 1));
    act_[w].desc = A.alloc<int4>(std::max<int64_t>(T[w]->nwc, 1));
    {  // cone records in cone order (SOC list, then RSOC list, as the cone tables)
      const std::vector<int64_t>& soc = w ? h_socG_ : h_socx_;
      const std::vector<int64_t>& rsoc = w ? h_rsocG_ : h_rsocx_;
      std::vector<int4>& cd = cone_desc_[w];
      cd.assign(T[w]->nwc, make_int4(0, 0, 0, 0));
      int64_t st = w ? (int64_t)(P.mGzero + P.mGnonnegative) : nb_;
      int64_t i = 0;
      for (const std::vector<int64_t>* L : {&soc, &rsoc})
        for (int64_t d : *L) {
          cd[i] = make_int4((int32_t)st, (int32_t)(d | (L == &rsoc ? (1 << 30) : 0)), (int32_t)i, 0);
          st += d;
          ++i;
        }
      for (int64_t k = 0; k < K_; ++k) {
        const std::array<int64_t, 8>& c = cones_[w][k];
        for (int64_t q = c[0]; q < c[1]; ++q) cd[q].w = (int32_t)k;
        for (int64_t q = c[2]; q < c[3]; ++q) cd[q].w = (int32_t)k;
      }
    }
    act_[w].exp = A.alloc<int32_t>(std::max<int64_t>(ne, 1));
    bytes += nc * sizeof(int2) + (2 * kCls + 4) * sizeof(int64_t) + T[w]->nwc * (sizeof(int64_t) + sizeof(int4)) +
             ne * sizeof(int32_t) + 256;
  }
  rchunk_ = A.alloc<int4>(std::max<int64_t>(nr, 1));
  n_rchunk_ = A.alloc<int64_t>(1);
  act_inst_ = A.alloc<int32_t>(K_);
  n_act_ = A.alloc<int64_t>(1);
  bytes += nr * sizeof(int4) + K_ * sizeof(int32_t) + 2 * sizeof(int64_t) + 16 * 256;
  if (tiled_) bytes += (size_t)(tl_[0].T.ntiles + tl_[1].T.ntiles) * sizeof(int32_t) + 4 * 256;
  act_bytes_ = bytes;
  const size_t need = pin_cap_ + bytes;
  PDCS_CUDA(cudaStreamSynchronize(s_));
  PDCS_CUDA(cudaFreeHost(pin_));
  pin_ = nullptr;
  PDCS_CUDA(cudaMallocHost(&pin_, need));
  pin_cap_ = need;
  pin_off_ = 0;
  XIg_ = XI;
  XIg_.act_chunk = act_[0].chunk;
  XIg_.act_meta = act_[0].meta;
  XIg_.act_sched = act_[0].sched;
  XIg_.act_exp = act_[0].exp;
  XIg_.act_desc = act_[0].desc;
  YIg_ = YI;
  YIg_.act_chunk = act_[1].chunk;
  YIg_.act_meta = act_[1].meta;
  YIg_.act_sched = act_[1].sched;
  YIg_.act_exp = act_[1].exp;
  YIg_.act_desc = act_[1].desc;
}

// Lists of the work of the iterating instances: elementwise chunks, warp cones
// by size class, exp cones, reflection chunks and the instances themselves.
void BatchSolver::build_act_lists(const std::vector<Inst*>& its) {
  std::vector<uint8_t> set(K_, 0);
  for (Inst* I : its) set[I->k] = 1;
  if (set == act_set_) return;
  act_set_ = set;
  auto chunks = [](int64_t start, int64_t len, auto&& emit) {
    for (int64_t o = 0; o < len; o += kThreads) emit(start + o, std::min<int64_t>(kThreads, len - o));
  };
  for (int w = 0; w < 2; ++w) {
    const std::vector<int64_t>& rs = w ? yrun_start_ : xrun_start_;
    const std::vector<int64_t>& rl = w ? yrun_len_ : xrun_len_;
    std::vector<int2> ch;
    std::vector<int64_t> bycls[kCls];
    std::vector<int32_t> ex;
    for (Inst* I : its) {
      const int64_t k = I->k;
      for (int q = 0; q < (w ? 2 : 1); ++q)  // elementwise runs: x box; y zero, nonneg
        chunks(rs[k * kMaxRuns + q], rl[k * kMaxRuns + q],
               [&](int64_t a, int64_t l) { ch.push_back(make_int2((int32_t)a, (int32_t)l)); });
      const std::array<int64_t, 8>& c = cones_[w][k];
      for (int64_t i = c[0]; i < c[1]; ++i) bycls[cone_cls_[w][i]].push_back(i);
      for (int64_t i = c[2]; i < c[3]; ++i) bycls[cone_cls_[w][i]].push_back(i);
      for (int64_t i = c[4]; i < c[5]; ++i) ex.push_back((int32_t)i);
      for (int64_t i = c[6]; i < c[7]; ++i) ex.push_back((int32_t)i);
    }
    int64_t* meta = stage<int64_t>(2 * kCls + 4);
    meta[0] = (int64_t)ch.size();
    int64_t task = 0, off = 0;
    size_t total = 0;
    for (int c = 0; c < kCls; ++c) total += bycls[c].size();
    int64_t* sched = stage<int64_t>(std::max<size_t>(total, 1));
    int4* desc = stage<int4>(std::max<size_t>(total, 1));
    for (int c = 0; c < kCls; ++c) {
      meta[1 + c] = task;
      meta[kCls + 2 + c] = off;
      std::memcpy(sched + off, bycls[c].data(), bycls[c].size() * sizeof(int64_t));
      for (size_t q = 0; q < bycls[c].size(); ++q) desc[off + q] = cone_desc_[w][bycls[c][q]];
      const int64_t per = (c < kCls - 1) ? 32 / cls_lanes(c) : 1;
      task += ((int64_t)bycls[c].size() + per - 1) / per;
      off += (int64_t)bycls[c].size();
    }
    meta[1 + kCls] = task;
    meta[2 * kCls + 2] = off;
    meta[2 * kCls + 3] = (int64_t)ex.size();
    PDCS_CUDA(cudaMemcpyAsync(act_[w].meta, meta, sizeof(int64_t) * (2 * kCls + 4), cudaMemcpyHostToDevice, s_));
    if (total) {
      PDCS_CUDA(cudaMemcpyAsync(act_[w].sched, sched, sizeof(int64_t) * total, cudaMemcpyHostToDevice, s_));
      PDCS_CUDA(cudaMemcpyAsync(act_[w].desc, desc, sizeof(int4) * total, cudaMemcpyHostToDevice, s_));
    }
    if (!ch.empty()) {
      int2* hc = stage<int2>(ch.size());
      std::memcpy(hc, ch.data(), ch.size() * sizeof(int2));
      PDCS_CUDA(cudaMemcpyAsync(act_[w].chunk, hc, sizeof(int2) * ch.size(), cudaMemcpyHostToDevice, s_));
    }
    if (!ex.empty()) {
      int32_t* he = stage<int32_t>(ex.size());
      std::memcpy(he, ex.data(), ex.size() * sizeof(int32_t));
      PDCS_CUDA(cudaMemcpyAsync(act_[w].exp, he, sizeof(int32_t) * ex.size(), cudaMemcpyHostToDevice, s_));
    }
  }
  std::vector<int4> rc;
  for (Inst* I : its)
    for (int w = 0; w < 2; ++w) {
      const std::vector<int64_t>& rs = w ? yrun_start_ : xrun_start_;
      const std::vector<int64_t>& rl = w ? yrun_len_ : xrun_len_;
      for (int q = 0; q < kMaxRuns; ++q)
        chunks(rs[I->k * kMaxRuns + q], rl[I->k * kMaxRuns + q],
               [&](int64_t a, int64_t l) { rc.push_back(make_int4((int32_t)a, (int32_t)l, w, (int32_t)I->k)); });
    }
  int64_t* hn = stage<int64_t>(2);
  hn[0] = (int64_t)rc.size();
  hn[1] = (int64_t)its.size();
  PDCS_CUDA(cudaMemcpyAsync(n_rchunk_, hn, sizeof(int64_t), cudaMemcpyHostToDevice, s_));
  PDCS_CUDA(cudaMemcpyAsync(n_act_, hn + 1, sizeof(int64_t), cudaMemcpyHostToDevice, s_));
  if (!rc.empty()) {
    int4* hr = stage<int4>(rc.size());
    std::memcpy(hr, rc.data(), rc.size() * sizeof(int4));
    PDCS_CUDA(cudaMemcpyAsync(rchunk_, hr, sizeof(int4) * rc.size(), cudaMemcpyHostToDevice, s_));
  }
  int32_t* hi = stage<int32_t>(std::max<size_t>(its.size(), 1));
  for (size_t i = 0; i < its.size(); ++i) hi[i] = (int32_t)its[i]->k;
  PDCS_CUDA(cudaMemcpyAsync(act_inst_, hi, sizeof(int32_t) * its.size(), cudaMemcpyHostToDevice, s_));
  if (fused_)
    for (int w = 0; w < 2; ++w) {  // the iterating instances' fused tiles, largest first
      const Fused& f = fu_[w];
      size_t cnt = 0;
      for (Inst* I : its) cnt += (size_t)(f.first[I->k + 1] - f.first[I->k]);
      int32_t* ht = stage<int32_t>(std::max<size_t>(cnt, 1));
      int64_t* hnt = stage<int64_t>(1);
      size_t j = 0;
      for (Inst* I : its)
        for (int64_t q = f.first[I->k]; q < f.first[I->k + 1]; ++q) ht[j++] = (int32_t)q;
      std::stable_sort(ht, ht + cnt, [&](int32_t a, int32_t b) { return f.nnz[a] > f.nnz[b]; });
      hnt[0] = (int64_t)cnt;
      PDCS_CUDA(cudaMemcpyAsync(const_cast<int32_t*>(f.F.act), ht, sizeof(int32_t) * cnt, cudaMemcpyHostToDevice, s_));
      PDCS_CUDA(cudaMemcpyAsync(const_cast<int64_t*>(f.F.n_act), hnt, sizeof(int64_t), cudaMemcpyHostToDevice, s_));
    }
  if (tiled_)
    for (int w = 0; w < 2; ++w) {  // the iterating instances' tiles, largest first
      const Tiles& t = tl_[w];
      size_t cnt = 0;
      for (Inst* I : its) cnt += (size_t)(t.first[I->k + 1] - t.first[I->k]);
      int32_t* ht = stage<int32_t>(std::max<size_t>(cnt, 1));
      int64_t* hnt = stage<int64_t>(1);
      size_t j = 0;
      for (Inst* I : its)
        for (int64_t q = t.first[I->k]; q < t.first[I->k + 1]; ++q) ht[j++] = (int32_t)q;
      std::stable_sort(ht, ht + cnt, [&](int32_t a, int32_t b) { return t.nnz[a] > t.nnz[b]; });
      hnt[0] = (int64_t)cnt;
      PDCS_CUDA(cudaMemcpyAsync(const_cast<int32_t*>(t.T.act), ht, sizeof(int32_t) * cnt, cudaMemcpyHostToDevice, s_));
      PDCS_CUDA(cudaMemcpyAsync(const_cast<int64_t*>(t.T.n_act), hnt, sizeof(int64_t), cudaMemcpyHostToDevice, s_));
    }
}

// Rebuild the iteration graph's row lists from the rows of the masked instances.
void BatchSolver::compact(const uint8_t* mask) {
  const CsrDev* full[2] = {&G_, &Gt_};
  for (int w = 0; w < 2; ++w) {
    Compact& c = cmp_[w];
    const int64_t R = full[w]->bin_off[kBins];
    row_flags_kernel<<<grid_for(R + 1), kThreads, 0, s_>>>(full[w]->rows, R, mask, c.flag);
    PDCS_CUDA(cub::DeviceScan::ExclusiveSum(c.tmp, c.tmp_bytes, c.flag, c.pos, (int)(R + 1), s_));
    row_compact_kernel<<<grid_for(R), kThreads, 0, s_>>>(full[w]->rows, R, c.flag, c.pos, c.rows, c.full_bin,
                                                         c.cbin);
    kernels_ += 3;
  }
}

namespace {
// a copy of A's schedule with at most cap CTAs per row bin (the kernel loops over its bin's rows)
template <class T>
CsrT<T> capped_bins(const CsrT<T>& A, int cap) {
  CsrT<T> B = A;
  B.cta0[0] = 0;
  for (int b = 0; b < kBins; ++b) B.cta0[b + 1] = B.cta0[b] + std::min(A.cta0[b + 1] - A.cta0[b], cap);
  return B;
}
// a copy of T with at most cap CTAs per part (every part loops over its work)
ConeTable capped_parts(const ConeTable& T, int cap) {
  ConeTable C = T;
  C.ctaA = std::min(T.ctaA, cap);
  C.ctaB = std::min(T.ctaB, cap);
  C.ctaC = std::min(T.ctaC, cap);
  return C;
}
}  // namespace

void BatchSolver::capture_batch_graph(int tail) {
  const int bin_cap = tail ? kTailBinCtas : INT32_MAX, cap = tail ? kTailCtas : INT32_MAX;
  const CsrT<float> G32 = capped_bins(G32c_, bin_cap), Gt32 = capped_bins(Gt32c_, bin_cap);
  const CsrDev G = capped_bins(Gc_, bin_cap), Gt = capped_bins(Gtc_, bin_cap);
  const ConeTable XI = capped_parts(XIg_, cap), YI = capped_parts(YIg_, cap);
  const int ctl_grid = tail ? (int)std::max<int64_t>(1, std::min<int64_t>(K_, cap))
                            : (int)std::max<int64_t>(1, std::min<int64_t>((K_ * 32 + kThreads - 1) / kThreads, 148 * 16));
  const int refl_grid = std::min(grid_reflect_, cap);
  const int tgrid[2] = {std::min(tl_[0].grid, cap), std::min(tl_[1].grid, cap)};
  const bool timed = O.verbose >= 2;
  if (timed)
    for (cudaEvent_t& e : gev_[tail])
      if (!e) PDCS_CUDA(cudaEventCreate(&e));
  PDCS_CUDA(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal));
  for (int a = 0; a < attempts_per_graph_; ++a) {
    int32_t* cur = live_cnt_ + (a & 1);
    int32_t* nxt = live_cnt_ + ((a + 1) & 1);
    const bool ev = timed && a == attempts_per_graph_ - 1;
    auto mark = [&](int i) {
      if (ev) PDCS_CUDA(cudaEventRecordWithFlags(gev_[tail][i], s_, cudaEventRecordExternal));  // a node of the graph
    };
    BatchCtl ctl{sts_, ps_,   ds_,     live_,      rx_,  ry_,         dxsq_,    dysq_,
                 dgdy_, cur,  nxt,     done_ctas_, live_cnt_ + 2, act_inst_, n_act_};
    mark(0);
    if (fused_ && !tail) {
      // two fused tile kernels: G' rows (primal step), then G rows (dual step)
      ctl.tpx = fu_[1].tpart;
      ctl.tpy = fu_[0].tpart;
      ctl.tfx = fu_[1].first_dev;
      ctl.tfy = fu_[0].first_dev;
      if (fp32_) {
        launch_fused<float, 1>(fu_[1].F, fu_[1].grid, fu_[1].sv32, dyl32_, nullptr,
                               FusedPrimal32{xa_, dxp32_, qa_, ps_, live_}, XIg_, fu_[1].tpart, cur, s_);
        mark(1);
        mark(2);
        launch_fused<float, kPair>(fu_[0].F, fu_[0].grid, fu_[0].sv32, &dxp32_->x, nullptr,
                                   FusedDual32{ya_, dyl32_, ra_, dy32_, ds_, live_}, YIg_, fu_[0].tpart, cur, s_);
      } else {
        launch_fused<double, 1>(fu_[1].F, fu_[1].grid, fu_[1].sv64, yl, nullptr,
                                FusedPrimal64{xl, c_s, x, ps_, live_}, XIg_, fu_[1].tpart, cur, s_);
        mark(1);
        mark(2);
        launch_fused<double, 2>(fu_[0].F, fu_[0].grid, fu_[0].sv64, x, xl,
                                FusedDual64{yl, h_s, y, ds_, live_}, YIg_, fu_[0].tpart, cur, s_);
      }
      mark(3);
    } else if (fp32_) {
      if (tiled_ && !tail) launch_spmv_tile<float, 1>(tl_[1].T, tgrid[1], Gt32_.v, dyl32_, nullptr, aty32_, nullptr, cur, s_);
      else launch_spmv<1, false, float>(Gt32, dyl32_, nullptr, aty32_, nullptr, cur, s_);
      mark(1);
      OpPrimalStep32B op1{xa_, dxp32_, qa_, aty32_, x, ix_, live_, ps_, dxsq_};
      launch_update_project(op1, XI, part_x, cur, s_);
      mark(2);
      if (tiled_ && !tail)
        launch_spmv_tile<float, kPair>(tl_[0].T, tgrid[0], G32_.v, &dxp32_->x, nullptr, gx32_, gxl32_, cur, s_);
      else launch_spmv<kPair, false, float>(G32, &dxp32_->x, nullptr, gx32_, gxl32_, cur, s_);
      mark(3);
      OpDualStep32B op2{ya_, dyl32_, ra_, gx32_, gxl32_, dy32_, y, iy_, live_, ds_, dysq_, dgdy_};
      launch_update_project(op2, YI, part_y, cur, s_);
    } else {
      if (tiled_ && !tail) launch_spmv_tile<double, 1>(tl_[1].T, tgrid[1], Gt_.v, yl, nullptr, aty, nullptr, cur, s_);
      else launch_spmv<1>(Gt, yl, nullptr, aty, nullptr, cur, s_);
      mark(1);
      OpPrimalStepB op1{xl, aty, c_s, x, ix_, live_, ps_, dxsq_};
      launch_update_project(op1, XI, part_x, cur, s_);
      mark(2);
      if (tiled_ && !tail) launch_spmv_tile<double, 2>(tl_[0].T, tgrid[0], G_.v, x, xl, gx, gxl, cur, s_);
      else launch_spmv<2>(G, x, xl, gx, gxl, cur, s_);
      mark(3);
      OpDualStepB op2{yl, gx, gxl, h_s, y, iy_, live_, ds_, dysq_, dgdy_};
      launch_update_project(op2, YI, part_y, cur, s_);
    }
    mark(4);
    if (tail) batch_control_kernel<true><<<ctl_grid, kThreads, 0, s_>>>(K_, ctl);
    else batch_control_kernel<false><<<ctl_grid, kThreads, 0, s_>>>(K_, ctl);
    mark(5);
    if (fp32_)
      batch_reflect32_kernel<<<refl_grid, kThreads, 0, s_>>>(cur, sts_, dxp32_, dxm_, dy32_, dyl32_, dym_, rchunk_,
                                                             n_rchunk_);
    else
      batch_reflect_kernel<<<refl_grid, kThreads, 0, s_>>>(cur, sts_, x, xl, xm, y, yl, ym, rchunk_, n_rchunk_);
    mark(6);
  }
  PDCS_CUDA(cudaStreamEndCapture(s_, &bgraph_[tail]));
  PDCS_CUDA(cudaGraphInstantiate(&bgraph_exec_[tail], bgraph_[tail], 0));
}

// Run one batched operation for a group of instances with identical requests.
void BatchSolver::exec_group(std::vector<Inst*>& g) {
  const ReqPayload& q = g[0]->req.key;
  rounds_++;
  const uint8_t* mask = upload_mask(g);
  auto kresid_side = [&](SegSide& S, double* contrib, int64_t stride) {
    const int32_t kinds[7] = {SK_SUM, SK_MAX, SK_MAX, SK_SUM, SK_MAX, SK_SUM, SK_SUM};  // OpResidual's kResid7
    for (int r = 0; r < 7; ++r) {
      S.a[r] = contrib + r * stride;
      S.kind[r] = kinds[r];
    }
  };
  switch (q.type) {
    case RQ_LIN: {
      LinList L{};
      for (int i = 0; i < q.count; ++i) L.op[i] = q.lin[i];
      L.count = q.count;
      masked_lin_kernel<<<grid_for(std::max(n_, m_)), kThreads, 0, s_>>>(L, ix_, iy_, mask, n_, m_);
      kernels_++;
      break;
    }
    case RQ_SPMV: {
      spmv_masked(q.side ? Gt_ : G_, q.p[0], const_cast<double*>(q.p[1]), mask);
      break;
    }
    case RQ_REFLECT: {
      PdhgState* h = stage<PdhgState>(K_);
      for (int64_t k = 0; k < K_; ++k) h[k] = inst_[k].S;
      PDCS_CUDA(cudaMemcpyAsync(sts_, h, sizeof(PdhgState) * K_, cudaMemcpyHostToDevice, s_));
      masked_reflect_kernel<<<grid_reflect_, kThreads, 0, s_>>>(sts_, ix_, iy_, mask, x, xl, xm, n_, y, yl, ym, m_);
      kernels_++;
      break;
    }
    case RQ_CONVERGE: {
      const double *xs = q.p[0], *ys = q.p[1];
      double *gxs = const_cast<double*>(q.p[2]), *atys = const_cast<double*>(q.p[3]);
      if (q.side == 0) {  // side 1: the products G xs, G' ys are given
        spmv_masked(G_, xs, gxs, mask);
        spmv_masked(Gt_, ys, atys, mask);
      }
      PerElem<OpResidual> opp{OpResidual{gxs, Dl, 1.0, nullptr, 0.0, h_raw, tm[5], bl_fin, bu_fin, 0}, tm[5], cy_, m_,
                              iy_, mask};
      update_project(opp, CON, part_a);
      PerElem<OpResidual> opd{OpResidual{atys, Dr, -1.0, c_raw, 1.0, nullptr, tn[5], bl_fin, bu_fin, nb_}, tn[5], cx_,
                              n_, ix_, mask};
      update_project(opd, SLK, part_b);
      SegSide X{}, Y{};
      kresid_side(X, cx_, n_);
      X.a[7] = c_raw; X.b[7] = xs; X.sa[7] = Dr; X.kind[7] = SK_DOT;
      X.count = 8;
      kresid_side(Y, cy_, m_);
      Y.a[7] = h_raw; Y.b[7] = ys; Y.sa[7] = Dl; Y.kind[7] = SK_DOT;
      Y.count = 8;
      seg_launch(mask, X, Y, 16);
      const double* r = seg_fetch(16);
      for (Inst* I : g) {
        const double* v = r + I->k * 16;
        // single-solver layout: [0..6] primal residual (y side), [7..13] dual (x side), 14 c'x, 15 h'y
        for (int i = 0; i < 7; ++i) {
          I->req.out[i] = v[8 + i];
          I->req.out[7 + i] = v[i];
        }
        I->req.out[14] = v[7];
        I->req.out[15] = v[15];
      }
      break;
    }
    case RQ_PROBE: {
      // p: px, py, h1, h2, gpx, xs, ys, gxs; s0 / s1: per-instance steps
      double* a0 = stage<double>(K_);
      double* a1 = stage<double>(K_);
      for (Inst* I : g) {
        a0[I->k] = I->req.s0;
        a1[I->k] = I->req.s1;
      }
      PDCS_CUDA(cudaMemcpyAsync(s0_, a0, sizeof(double) * K_, cudaMemcpyHostToDevice, s_));
      PDCS_CUDA(cudaMemcpyAsync(s1_, a1, sizeof(double) * K_, cudaMemcpyHostToDevice, s_));
      double *xs = const_cast<double*>(q.p[5]), *ys = const_cast<double*>(q.p[6]);
      double* gxs = const_cast<double*>(q.p[7]);
      PerElem<OpAxpyProjB> ox{OpAxpyProjB{q.p[0], q.p[2], s0_, xs, nullptr, nullptr, ix_}, xs, cx_, n_, ix_, mask};
      update_project(ox, XI, part_a);
      spmv_masked(G_, xs, gxs, mask);
      PerElem<OpAxpyProjB> oy{OpAxpyProjB{q.p[1], q.p[3], s1_, ys, gxs, q.p[4], iy_}, ys, cy_, m_, iy_, mask};
      update_project(oy, YI, part_b);
      SegSide X{}, Y{};
      X.a[0] = cx_; X.kind[0] = SK_SUM;
      X.a[1] = cx_ + n_; X.kind[1] = SK_SUM;
      X.count = 2;
      Y.a[0] = cy_; Y.kind[0] = SK_SUM;
      Y.a[1] = cy_ + m_; Y.kind[1] = SK_SUM;
      Y.a[2] = cy_ + 2 * m_; Y.kind[2] = SK_SUM;
      Y.count = 3;
      seg_launch(mask, X, Y, 5);
      const double* r = seg_fetch(5);
      for (Inst* I : g) {
        const double* v = r + I->k * 5;
        I->req.out[0] = v[0];
        I->req.out[1] = v[1];
        I->req.out[3] = v[2];
        I->req.out[4] = v[3];
        I->req.out[5] = v[4];
      }
      break;
    }
    case RQ_BSEARCH: {
      double* prm = stage<double>(4 * K_);
      int32_t* list = stage<int32_t>(g.size());
      for (size_t i = 0; i < g.size(); ++i) {
        const Inst* I = g[i];
        list[i] = (int32_t)I->k;
        prm[4 * I->k] = I->req.s0;
        prm[4 * I->k + 1] = I->req.s1;
        prm[4 * I->k + 2] = I->req.s2;
        prm[4 * I->k + 3] = I->req.s3;
      }
      PDCS_CUDA(cudaMemcpyAsync(bs_prm_, prm, sizeof(double) * 4 * K_, cudaMemcpyHostToDevice, s_));
      PDCS_CUDA(cudaMemcpyAsync(bs_list_, list, sizeof(int32_t) * g.size(), cudaMemcpyHostToDevice, s_));
      BsArgs B{};
      B.list = bs_list_;
      B.rx = rx_;
      B.ry = ry_;
      B.cones_x = cones_dev_[0];
      B.cones_y = cones_dev_[1];
      B.X = XI;
      B.Y = YI;
      B.G = G_;
      B.Gt = Gt_;
      B.c = c_s;
      B.h = h_s;
      B.h1 = tn[2];
      B.h2 = tm[2];
      B.xs = tn[3];
      B.ys = tm[3];
      B.gpx = tm[1];
      B.gxs = tm[4];
      B.nsearch = q.count;
      for (int i = 0; i < q.count; ++i) {
        B.px[i] = q.p[2 * i];
        B.py[i] = q.p[2 * i + 1];
      }
      B.prm = bs_prm_;
      B.out = bs_out_;
      bsearch_kernel<<<(int)g.size(), kThreads, 0, s_>>>(B);
      kernels_++;
      double* o = stage<double>(5 * K_);
      PDCS_CUDA(cudaMemcpyAsync(o, bs_out_, sizeof(double) * 5 * K_, cudaMemcpyDeviceToHost, s_));
      sync_reset();
      for (Inst* I : g)
        for (int i = 0; i < 5; ++i) I->req.out[i] = o[5 * I->k + i];
      break;
    }
    case RQ_MNORM: {
      double* gdx = const_cast<double*>(q.p[2]);
      spmv_masked(G_, q.p[0], gdx, mask);
      SegSide X{}, Y{};
      X.a[0] = q.p[0]; X.kind[0] = SK_DOT;
      X.count = 1;
      Y.a[0] = q.p[1]; Y.b[0] = gdx; Y.kind[0] = SK_DOT;
      Y.a[1] = q.p[1]; Y.kind[1] = SK_DOT;
      Y.count = 2;
      seg_launch(mask, X, Y, 3);
      const double* r = seg_fetch(3);
      for (Inst* I : g) {
        const double* v = r + I->k * 3;
        I->req.out[0] = v[1];
        I->req.out[1] = v[2];
        I->req.out[2] = v[0];
      }
      break;
    }
    case RQ_SEG: {
      const int stride = q.X.count + q.Y.count;
      seg_launch(mask, q.X, q.Y, stride);
      const double* r = seg_fetch(stride);
      for (Inst* I : g)
        for (int i = 0; i < stride; ++i) I->req.out[i] = r[I->k * stride + i];
      break;
    }
    default:
      throw std::logic_error("unknown batch request");
  }
}

// Run shared graphs of PDHG attempts until some iterating instance halts.
void BatchSolver::exec_iterate(std::vector<Inst*>& its) {
  Timer tm_(t_iter_);
  if (!bgraph_exec_[0]) {
    capture_batch_graph(0);
    capture_batch_graph(1);
  }
  std::vector<uint8_t> iterating(K_, 0);
  for (Inst* I : its) iterating[I->k] = 1;
  PdhgState* hs = stage<PdhgState>(K_);
  double* hps = stage<double>(K_);
  double* hds = stage<double>(K_);
  uint8_t* hl = stage<uint8_t>(K_);
  int32_t* hc = stage<int32_t>(4);
  int64_t to_check = 1 << 20;
  for (int64_t k = 0; k < K_; ++k) {
    PdhgState s = inst_[k].S;
    s.active = iterating[k] ? 1 : 0;
    s.do_reflect = 0;
    hs[k] = s;
    hps[k] = s.ps;
    hds[k] = s.ds;
    hl[k] = (uint8_t)s.active;
    if (iterating[k] && s.check_freq > 0) to_check = std::min<int64_t>(to_check, s.check_freq - (s.iter % s.check_freq));
  }
  hc[0] = (int32_t)its.size();
  hc[1] = 0;
  hc[2] = 0;
  hc[3] = 0;
  PDCS_CUDA(cudaMemcpyAsync(sts_, hs, sizeof(PdhgState) * K_, cudaMemcpyHostToDevice, s_));
  PDCS_CUDA(cudaMemcpyAsync(ps_, hps, sizeof(double) * K_, cudaMemcpyHostToDevice, s_));
  PDCS_CUDA(cudaMemcpyAsync(ds_, hds, sizeof(double) * K_, cudaMemcpyHostToDevice, s_));
  PDCS_CUDA(cudaMemcpyAsync(live_, hl, K_, cudaMemcpyHostToDevice, s_));
  PDCS_CUDA(cudaMemcpyAsync(live_cnt_, hc, 4 * sizeof(int32_t), cudaMemcpyHostToDevice, s_));
  // the graph's SpMVs run over the rows of the iterating instances only (rows of
  // instances that halt during these graphs are still computed; their products
  // are not read before the next attempt or anchor recomputes them)
  int64_t live_nnz = 0;
  for (Inst* I : its) live_nnz += probs_[I->k].nnz;
  // the tail graph (few nonzeros left) runs the binned SpMV over compacted rows;
  // the full graph runs the instance tiles when the batch has them
  const int tail = (live_nnz < kTailNnz && 16 * live_nnz < nnz_) ? 1 : 0;
  int64_t max_nnz = 0;
  for (Inst* I : its) max_nnz = std::max<int64_t>(max_nnz, probs_[I->k].nnz);
  const bool cta_tail = tail && max_nnz <= kTailCtaNnz;
  if (!cta_tail && (!tiled_ || tail)) compact(live_);
  build_act_lists(its);
  if (fp32_) {
    // FP64 anchors at the current iterates: for instances that (re)start
    // iterating, and every round for the others (refinement keeps the FP32
    // deltas small: at most the movement of one round)
    std::vector<Inst*> again;
    for (Inst* I : its)
      if (I->anchored) again.push_back(I);
    if (!again.empty()) materialize(ix_, iy_, upload_mask(again));
    for (Inst* I : its) I->anchored = true;
    anchor(ix_, iy_, live_);
  }
  int64_t graphs = (to_check + attempts_per_graph_ - 1) / attempts_per_graph_;
  graphs = std::max<int64_t>(1, std::min<int64_t>(graphs, 4));
  const double t_round = now_s();
  if (O.verbose) {
    for (cudaEvent_t& e : round_ev_)
      if (!e) PDCS_CUDA(cudaEventCreate(&e));
    PDCS_CUDA(cudaEventRecord(round_ev_[0], s_));
  }
  if (cta_tail) {
    TailArgs T{};
    T.list = act_inst_;
    // the loop re-anchors by itself, so a tail round runs up to the next checkpoint
    T.max_attempts = (int32_t)std::max<int64_t>(graphs * attempts_per_graph_, std::min<int64_t>(to_check, 1 << 20));
    T.ctl = BatchCtl{sts_,   ps_,     ds_,         live_, rx_,    ry_,       dxsq_,  dysq_,
                     dgdy_,  nullptr, nullptr,     nullptr, nullptr, act_inst_, n_act_};
    T.X = XI;
    T.Y = YI;
    T.cones_x = cones_dev_[0];
    T.cones_y = cones_dev_[1];
    const int grid = (int)its.size();
    if (fp32_) {
      TailFP32 pk{Gt32_, G32_,
                  OpPrimalStep32B{xa_, dxp32_, qa_, aty32_, x, ix_, live_, ps_, dxsq_},
                  OpDualStep32B{ya_, dyl32_, ra_, gx32_, gxl32_, dy32_, y, iy_, live_, ds_, dysq_, dgdy_},
                  dxp32_, dxm_, dy32_, dyl32_, dym_, aty32_, gx32_, gxl32_,
                  Gt_, G_, x, xl, xm, y, yl, ym, xa_, ya_, qa_, ra_, c_s, h_s};
      tail_attempts_kernel<TailFP32><<<grid, kThreads, 0, s_>>>(T, pk);
    } else {
      TailFP64 pk{Gt_, G_, OpPrimalStepB{xl, aty, c_s, x, ix_, live_, ps_, dxsq_},
                  OpDualStepB{yl, gx, gxl, h_s, y, iy_, live_, ds_, dysq_, dgdy_},
                  x, xl, xm, y, yl, ym, aty, gx, gxl};
      tail_attempts_kernel<TailFP64><<<grid, kThreads, 0, s_>>>(T, pk);
    }
    PDCS_CUDA(cudaGetLastError());
    kernels_++;
    tail_rounds_++;
  } else {
    for (int64_t gi = 0; gi < graphs; ++gi) {
      PDCS_CUDA(cudaGraphLaunch(bgraph_exec_[tail], s_));
      graphs_++;
      kernels_ += 6LL * attempts_per_graph_;
    }
  }
  if (O.verbose) PDCS_CUDA(cudaEventRecord(round_ev_[1], s_));
  PdhgState* back = stage<PdhgState>(K_);
  PDCS_CUDA(cudaMemcpyAsync(back, sts_, sizeof(PdhgState) * K_, cudaMemcpyDeviceToHost, s_));
  sync_reset();  // `back` stays readable: nothing is staged before the loop below ends
  if (O.verbose) {
    float dev = 0.0f;
    PDCS_CUDA(cudaEventElapsedTime(&dev, round_ev_[0], round_ev_[1]));
    dev_ms_ += dev;
    if (O.verbose >= 2 && gev_[tail][0] && !cta_tail) {  // the kernels of the round's last attempt
      for (int i = 0; i < 6; ++i) {
        float e = 0.0f;
        PDCS_CUDA(cudaEventElapsedTime(&e, gev_[tail][i], gev_[tail][i + 1]));
        gev_ms_[tail][i] += e;
      }
      gev_n_[tail]++;
    }
    std::printf("[pdcs_b200 batch] %.3f s: %zu of %lld instances iterating, %lld attempts in %.3f ms (device %.3f ms)%s\n",
                now_s() - t_start_, its.size(), (long long)K_, (long long)(graphs * attempts_per_graph_),
                1e3 * (now_s() - t_round), dev, cta_tail ? " (tail kernel)" : tail ? " (tail graph)" : "");
  }
  const bool timeout = O.time_limit > 0 && now_s() - t_start_ > O.time_limit;
  std::vector<Inst*> halted;
  for (Inst* I : its) {
    I->S = back[I->k];
    I->S.do_reflect = 0;  // applied by the graph's reflection kernel
    I->S.done_ctas = 0;
    if (!I->S.active || timeout) halted.push_back(I);
  }
  if (fp32_ && !halted.empty()) {  // their host requests work on the FP64 iterates
    materialize(ix_, iy_, upload_mask(halted));
    for (Inst* I : halted) I->anchored = false;
  }
  for (Inst* I : halted) resume(*I);
}

void BatchSolver::schedule() {
  for (auto& I : inst_) I.task = main_task(I);
  for (auto& I : inst_) {
    I.task.start();
    I.task.rethrow();
  }
  std::vector<Inst*> svc, its;
  while (true) {
    svc.clear();
    its.clear();
    for (auto& I : inst_) {
      if (I.task.done()) continue;
      if (I.req.key.type == RQ_ITERATE) its.push_back(&I);
      else svc.push_back(&I);
    }
    if (svc.empty() && its.empty()) break;
    if (!svc.empty()) {
      // group identical requests (hash buckets, verified byte-wise)
      std::unordered_map<uint64_t, std::vector<std::vector<Inst*>>> buckets;
      std::vector<std::vector<Inst*>*> order;
      for (Inst* I : svc) {
        auto& lists = buckets[I->req.hash];
        bool placed = false;
        for (auto& l : lists)
          if (std::memcmp(&l[0]->req.key, &I->req.key, sizeof(ReqPayload)) == 0) {
            l.push_back(I);
            placed = true;
            break;
          }
        if (!placed) lists.push_back({I});
      }
      for (auto& kv : buckets)
        for (auto& l : kv.second) order.push_back(&l);
      std::sort(order.begin(), order.end(), [](auto* a, auto* b) { return (*a)[0]->k < (*b)[0]->k; });
      for (auto* l : order) {
        const double t0 = now_s();
        const int32_t type = (*l)[0]->req.key.type & 15;
        exec_group(*l);
        for (Inst* I : *l) resume(*I);
        svc_s_[type] += now_s() - t0;
        svc_groups_[type]++;
        svc_insts_[type] += (int64_t)l->size();
      }
      continue;
    }
    const double t0 = now_s();
    exec_iterate(its);
    iter_s_ += now_s() - t0;
  }
}

// ---------------------------------------------------------------------------
// Per-instance algorithm: the single solver's main loop with device work
// expressed as requests.
// ---------------------------------------------------------------------------
Co<> BatchSolver::lin(Inst& I, std::vector<Lin> ops) {
  ReqPayload p = payload(RQ_LIN);
  for (const Lin& o : ops) {
    if (p.count == 6) {
      co_await post(I, p);
      p = payload(RQ_LIN);
    }
    LinOp& l = p.lin[p.count++];
    l.dst = o.dst;
    l.a = o.a;
    l.u = o.u;
    l.b = o.b;
    l.v = o.v;
    l.side = o.side;
  }
  if (p.count) co_await post(I, p);
}

Co<> BatchSolver::converge_info(Inst& I, const double* xs, const double* ys, Converge& C, double* gxs,
                                double* atys) {
  ReqPayload p = payload(RQ_CONVERGE);
  p.p[0] = xs;
  p.p[1] = ys;
  p.p[2] = gxs;
  p.p[3] = atys;
  co_await post(I, p);
  const double* r = I.req.out;
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
  C.l2_rel_p = l2p / (1.0 + std::max(snrm1, std::max(I.hNrm1, axnrm1)));
  C.linf_rel_p = linfp / (1.0 + std::max(sinf, std::max(I.hNrmInf, axinf)));
  C.l2_rel_d = l2d / (1.0 + std::max(I.cNrm1, atynrm1));
  C.linf_rel_d = linfd / (1.0 + std::max(I.cNrmInf, atyinf));
}

// exit_condition_check_diagonal! (rpdhg_alg_gpu_gen_scaling.jl:309-352) with the
// infeasibility information (:185-248), as Solver::exit_check
// the reference pushes the objective trends with probability 1/4
static void push_trend(const Inst& I, Infea& F) {
  if (I.check_count % 4 == 1) {
    F.ptrend.push_back(I.ci[0].pobj);
    F.dtrend.push_back(I.ci[0].dobj);
    if (F.ptrend.size() > 20) F.ptrend.erase(F.ptrend.begin());
    if (F.dtrend.size() > 20) F.dtrend.erase(F.dtrend.begin());
  }
}

Co<> BatchSolver::exit_check(Inst& I) {
  double *gxc = tm[0], *gxm = tm[1], *atc = tn[0], *atm = tn[1];
  co_await converge_info(I, x, y, I.ci[0], gxc, atc);
  co_await converge_info(I, xm, ym, I.ci[1], gxm, atm);
  I.check_count++;
  // ray = current - average; G and G' of the difference by linearity
  double *dxs = tn[2], *dys = tm[2], *gd = tm[3], *ad = tn[3];
  co_await lin(I, {{dxs, 1.0, x, -1.0, xm, 0}, {dys, 1.0, y, -1.0, ym, 1}, {gd, 1.0, gxc, -1.0, gxm, 1},
                   {ad, 1.0, atc, -1.0, atm, 0}});
  double nr[4];
  {
    // |x/Dr|_inf, |dx/Dr|_inf; |y/Dl|_inf, |dy/Dl|_inf
    ReqPayload s = payload(RQ_SEG);
    s.X.a[0] = x; s.X.sa[0] = Dr; s.X.kind[0] = SK_MAXABS;
    s.X.a[1] = dxs; s.X.sa[1] = Dr; s.X.kind[1] = SK_MAXABS;
    s.X.count = 2;
    s.Y.a[0] = y; s.Y.sa[0] = Dl; s.Y.kind[0] = SK_MAXABS;
    s.Y.a[1] = dys; s.Y.sa[1] = Dl; s.Y.kind[1] = SK_MAXABS;
    s.Y.count = 2;
    co_await post(I, s);
    for (int i = 0; i < 4; ++i) nr[i] = I.req.out[i];
  }
  {
    // residuals of the ray with its products given (gd = G dx, ad = G' dy)
    ReqPayload q = payload(RQ_CONVERGE);
    q.p[0] = dxs;
    q.p[1] = dys;
    q.p[2] = gd;
    q.p[3] = ad;
    q.side = 1;
    co_await post(I, q);
  }
  const double* r = I.req.out;
  {
    Infea& F = I.ii[0];
    F.primal_ray_obj = I.ci[0].pobj;
    F.dual_ray_obj = I.ci[0].dobj;
    F.max_primal_ray_inf = (I.ci[0].pobj < 0.0) ? I.ci[0].linf_abs_p : 1e10;
    F.max_dual_ray_inf = (I.ci[0].dobj > 0.0) ? I.ci[0].linf_abs_d : 1e10;
    F.primal_ray_norm = nr[0];
    F.dual_ray_norm = nr[2];
    push_trend(I, F);
  }
  {
    Infea& F = I.ii[1];
    double pobj = r[14];
    double dobj = r[15] + r[7 + 6];
    F.primal_ray_obj = pobj;
    F.dual_ray_obj = dobj;
    F.max_primal_ray_inf = (pobj < 0.0) ? r[1] : 1e10;
    F.max_dual_ray_inf = (dobj > 0.0) ? r[7 + 1] : 1e10;
    F.primal_ray_norm = nr[1];
    F.dual_ray_norm = nr[3];
    push_trend(I, F);
  }
  termination_check(I.ci, I.ii, I.S.iter, O, now_s() - t_start_, I.exit_code, I.pobj, I.dobj, I.returned_seq);
}

Co<double> BatchSolver::mnorm(Inst& I, const double* dx, const double* dy, double ta, double si) {
  ReqPayload p = payload(RQ_MNORM);
  p.p[0] = dx;
  p.p[1] = dy;
  p.p[2] = tm[4];
  co_await post(I, p);
  const double* r = I.req.out;
  co_return r[2] / ta - 2.0 * r[0] + r[1] / si;
}

Co<double> BatchSolver::binary_search(Inst& I, double r, const double* px, const double* py, double ta,
                                      double si) {
  double *h1 = tn[2], *h2 = tm[2], *xs = tn[3], *ys = tm[3], *gpx = tm[1], *gxs = tm[4];
  {
    ReqPayload a = payload(RQ_SPMV);
    a.side = 1;
    a.p[0] = py;
    a.p[1] = h1;
    co_await post(I, a);
    ReqPayload b = payload(RQ_SPMV);
    b.side = 0;
    b.p[0] = px;
    b.p[1] = gpx;
    co_await post(I, b);
  }
  co_await lin(I, {{h1, 1.0, h1, -1.0, c_s, 0}, {h2, -1.0, gpx, 1.0, h_s, 1}});
  double last_h1dx = 0.0, last_h2dy = 0.0;
  ReqPayload pr = payload(RQ_PROBE);
  pr.p[0] = px;
  pr.p[1] = py;
  pr.p[2] = h1;
  pr.p[3] = h2;
  pr.p[4] = gpx;
  pr.p[5] = xs;
  pr.p[6] = ys;
  pr.p[7] = gxs;
  double t = I.bs_t0, tR = t, tL = 0.0;
  for (int k = 1; k <= 1000; ++k) {
    double val = co_await approx(I, pr, ta, si, last_h1dx, last_h2dy, t);
    if (val > r && val < r + 1e-6) {
      tR = t;
      tL = std::max(t - 0.01, 0.0);
      val = co_await approx(I, pr, ta, si, last_h1dx, last_h2dy, tL);
      if (val < r) break;
    }
    if (val < r && val > r - 1e-6) {
      tL = t;
      tR = t + 0.01;
      val = co_await approx(I, pr, ta, si, last_h1dx, last_h2dy, tR);
      if (val > r) break;
    }
    if (val > r) break;
    t *= 2;
  }
  double tM = 0.5 * (tR + tL);
  int64_t count = 0;
  while (tR - tL > 1e-6) {
    tM = 0.5 * (tR + tL);
    const double v = co_await approx(I, pr, ta, si, last_h1dx, last_h2dy, tM);
    if (v < r) tL = tM;
    else tR = tM;
    if (++count > 1000000) break;
  }
  I.bs_t0 = tM;
  co_return (last_h1dx + last_h2dy) / r;
}

// The binary search(es) of one restart test on the device (bsearch_kernel):
// (px0, py0), then (px1, py1) when px1 is given, the second from the radius the
// first ends at.  Returns false, leaving bs_t0 as it was, when an instance's
// search needs more evaluations than the device path runs (the caller then
// runs binary_search).
Co<bool> BatchSolver::binary_search_dev(Inst& I, double r, const double* px0, const double* py0,
                                        const double* px1, const double* py1, double* vals) {
  ReqPayload p = payload(RQ_BSEARCH);
  p.count = px1 ? 2 : 1;
  p.p[0] = px0;
  p.p[1] = py0;
  p.p[2] = px1;
  p.p[3] = py1;
  co_await post(I, p, r, I.S.tau, I.S.sigma, I.bs_t0);
  const double* q = I.req.out;
  I.probes += (int64_t)q[0];
  probes_ += (int64_t)q[0];
  if (q[4] == 0.0) co_return false;
  I.bs_t0 = q[1];
  vals[0] = q[2];
  vals[1] = q[3];
  co_return true;
}

// one evaluation of the binary search at t (approx of Solver::binary_search)
Co<double> BatchSolver::approx(Inst& I, const ReqPayload& pr, double ta, double si, double& h1dx, double& h2dy,
                               double t) {
  I.probes++;
  probes_++;
  co_await post(I, pr, t * ta / 2, t * si / 2);
  const double* q = I.req.out;
  h1dx = q[1];
  h2dy = q[4];
  co_return q[0] / ta - 2.0 * q[5] + q[3] / si;
}

Co<> BatchSolver::restart_threshold(Inst& I, bool dgap) {
  if (dgap) {
    double *dx = tn[4], *dy = tm[5];
    co_await lin(I, {{dx, 1.0, x0, -1.0, x0l, 0}, {dy, 1.0, y0, -1.0, y0l, 1}});
    double r = co_await mnorm(I, dx, dy, I.S.tau, I.S.sigma);
    I.ndg_r = r;
    double v[2];
    if (co_await binary_search_dev(I, r, x0, y0, nullptr, nullptr, v)) I.ndg_thr = v[0];
    else I.ndg_thr = co_await binary_search(I, r, x0, y0, I.S.tau, I.S.sigma);
    if (I.ndg_thr < 0) I.dgap_flag = false;
  } else {
    co_await converge_info(I, x, y, I.ci[0], tm[0], tn[0]);
    I.kkt_thr = kkt_error_i(I, I.ci[0]);
  }
}

Co<bool> BatchSolver::restart_check(Inst& I, bool dgap) {
  if (dgap) {
    double *dx = tn[4], *dy = tm[5];
    co_await lin(I, {{dx, 1.0, x, -1.0, x0, 0}, {dy, 1.0, y, -1.0, y0, 1}});
    double rl = co_await mnorm(I, dx, dy, I.S.tau, I.S.sigma);
    double v[2], rho, rho_m;
    if (co_await binary_search_dev(I, rl, x, y, xm, ym, v)) {
      rho = v[0];
      rho_m = v[1];
    } else {
      rho = co_await binary_search(I, rl, x, y, I.S.tau, I.S.sigma);
      rho_m = co_await binary_search(I, rl, xm, ym, I.S.tau, I.S.sigma);
    }
    I.ndg[0] = rho;
    I.ndg[1] = rho_m;
    const double betas[2] = {0.4, 0.8};
    for (int bi = 0; bi < 2; ++bi) {
      const double beta = betas[bi];
      if (rho < beta * I.ndg_thr || rho_m < beta * I.ndg_thr) {
        I.restart_used++;
        if (I.ndg[0] < I.ndg[1] && I.dgap_flag) co_await lin(I, {{xm, 1.0, x, 0.0, nullptr, 0}, {ym, 1.0, y, 0.0, nullptr, 1}});
        co_return true;
      }
    }
  } else {
    co_await converge_info(I, x, y, I.ci[0], tm[0], tn[0]);
    co_await converge_info(I, xm, ym, I.ci[1], tm[1], tn[1]);
    double lag0 = I.kkt_err[0], lag1 = I.kkt_err[1];
    double e0 = kkt_error_i(I, I.ci[0]), e1 = kkt_error_i(I, I.ci[1]);
    I.kkt_err[0] = e0;
    I.kkt_err[1] = e1;
    bool c1 = e0 < 0.4 * I.kkt_thr || e1 < 0.4 * I.kkt_thr;
    bool c2 = (e0 < 0.8 * I.kkt_thr && e0 > lag0) || (e1 < 0.8 * I.kkt_thr && e1 > lag1);
    if (c1 || c2) {
      I.restart_used++;
      if (I.kkt_err[0] < I.kkt_err[1]) co_await lin(I, {{xm, 1.0, x, 0.0, nullptr, 0}, {ym, 1.0, y, 0.0, nullptr, 1}});
      co_return true;
    }
  }
  if ((double)I.S.inner >= (double)I.S.iter * 0.223 && I.S.iter > 100000) {
    I.restart_used++;
    co_return true;
  }
  co_return false;
}

Co<> BatchSolver::omega_update(Inst& I, const double* xds, const double* yds) {
  ReqPayload p = payload(RQ_SEG);
  p.X.a[0] = xds; p.X.b[0] = x; p.X.kind[0] = SK_DIFF2;
  p.X.count = 1;
  p.Y.a[0] = yds; p.Y.b[0] = y; p.Y.kind[0] = SK_DIFF2;
  p.Y.count = 1;
  co_await post(I, p);
  double xn = std::sqrt(I.req.out[0]), yn = std::sqrt(I.req.out[1]), om = I.S.omega;
  const int64_t ru = I.restart_used;
  if ((om > 1e4 || om < 1e-4) && ru % 20 == 0 && ru != 0) I.S.omega = I.omega0;
  else if ((om > 3e4 || om < 1.0 / 3e4) && ru % 10 == 0 && ru != 0) I.S.omega = I.omega0;
  else if (xn > 1e-10 && yn > 1e-10) I.S.omega = std::exp(0.5 * std::log(yn / xn) + 0.5 * std::log(om));
}

Co<> BatchSolver::iterate(Inst& I) {
  ReqPayload p = payload(RQ_ITERATE);
  co_await post(I, p);
}

Co<> BatchSolver::main_task(Inst& I) {
  PdhgState& S = I.S;
  co_await converge_info(I, x, y, I.ci[0], tm[0], tn[0]);  // rpdhg_alg_gpu_gen.jl:1865-1881
  co_await lin(I, {{x0, 1.0, x, 0.0, nullptr, 0}, {y0, 1.0, y, 0.0, nullptr, 1},
                   {x0l, 1.0, x, 0.0, nullptr, 0}, {y0l, 1.0, y, 0.0, nullptr, 1}});
  S = PdhgState{};
  S.omega = I.omega0;
  S.eta_p = 1.0 / I.ginf;
  S.tau = 0.9;
  S.sigma = 0.9;
  S.check_freq = O.check_terminate_freq;
  S.attempt_limit = O.attempt_limit;
  int64_t rf = 0;
  if (O.use_duality_gap_restart) rf = O.duality_gap_restart_freq;
  if (O.use_kkt_restart) rf = rf ? std::min(rf, O.kkt_restart_freq) : O.kkt_restart_freq;
  S.restart_freq = rf;
  S.restart_enabled = rf > 0;
  for (int64_t outer = 1; outer <= O.max_outer_iter; ++outer) {
    const bool bx = I.ci[0].l2_rel_p < I.pres_best, by = I.ci[0].l2_rel_d < I.dres_best;
    if (bx) I.pres_best = I.ci[0].l2_rel_p;
    if (by) I.dres_best = I.ci[0].l2_rel_d;
    if (bx && by) co_await lin(I, {{xbest, 1.0, x, 0.0, nullptr, 0}, {ybest, 1.0, y, 0.0, nullptr, 1}});
    else if (bx) co_await lin(I, {{xbest, 1.0, x, 0.0, nullptr, 0}});
    else if (by) co_await lin(I, {{ybest, 1.0, y, 0.0, nullptr, 1}});
    I.max_kkt = std::max(std::max(I.ci[0].l2_rel_p, I.ci[0].l2_rel_d), I.ci[0].rel_gap);
    I.min_kkt = std::min(std::min(std::min(I.ci[0].l2_rel_p, I.ci[0].l2_rel_d), I.ci[0].rel_gap), I.min_kkt);
    double extra = -0.1 * std::log10(I.max_kkt) + 0.2;
    co_await lin(I, {{x0l, 1.0, x0, 0.0, nullptr, 0}, {y0l, 1.0, y0, 0.0, nullptr, 1},
                     {x0, 1.0, xm, 0.0, nullptr, 0}, {y0, 1.0, ym, 0.0, nullptr, 1},
                     {x, 1.0, xm, 0.0, nullptr, 0}, {y, 1.0, ym, 0.0, nullptr, 1}});
    if (O.use_kkt_restart) co_await restart_threshold(I, false);
    else co_await restart_threshold(I, I.dgap_flag);
    {
      double pd = I.ci[0].l2_rel_p / I.ci[0].l2_rel_d;
      bool f1 = outer > 10 && I.max_kkt > 1e5;
      bool f2 = outer > 80 && (pd > 1e10 || pd < 1e-10);
      bool f3 = outer > 10 && S.tau < 1e-6 && S.sigma < 1e-6;
      bool f4 = S.iter > 1000000 && I.ci[0].rel_gap > 0.98 && I.ci[0].l2_rel_p > 1.0 && I.ci[0].l2_rel_d > 1.0;
      if (f1 || f2 || f3 || f4 || O.force_resolving) {
        I.needs_single = true;  // resolving fallback: the instance is re-solved on its own
        co_return;
      }
    }
    co_await lin(I, {{xl, 1.0, x, 0.0, nullptr, 0}, {yl, 1.0, y, 0.0, nullptr, 1},
                     {xds_, 1.0, x, 0.0, nullptr, 0}, {yds_, 1.0, y, 0.0, nullptr, 1}});
    S.inner = 0;
    S.eta_cum = 0.0;
    S.extra = extra;
    S.dec = std::min(0.9 + 0.1 * std::log10(I.max_kkt * 1e5), 1.0);
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
      co_await iterate(I);
      if (O.time_limit > 0 && now_s() - t_start_ > O.time_limit && S.active) {
        I.exit_code = PDCS_EXIT_TIME_LIMIT;
        co_return;
      }
      int reason = S.halt_reason;
      S.halt_reason = HALT_NONE;
      if (reason == HALT_LIMIT) {
        I.exit_code = PDCS_EXIT_ATTEMPT_LIMIT;
        co_return;
      }
      if (reason == HALT_CHECK) {
        co_await exit_check(I);
        I.max_kkt = std::max(std::max(I.ci[0].l2_rel_p, I.ci[0].l2_rel_d), I.ci[0].rel_gap);
        S.dec_next = std::min(0.9 + 0.1 * std::log10(I.max_kkt * 1e5), 1.0);
        if (I.exit_code != PDCS_EXIT_CONTINUE) co_return;
        if (S.attempt_limit > 0 && S.iter >= S.attempt_limit) {
          I.exit_code = PDCS_EXIT_ATTEMPT_LIMIT;
          co_return;
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
          co_await post(I, payload(RQ_REFLECT));
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
        I.restart_used++;
        restart = true;
        break;
      }
      if (reason == HALT_RESTART_CHECK) {
        bool brk = false;
        if (O.use_kkt_restart && O.kkt_restart_freq > 0 && S.iter % O.kkt_restart_freq == 0) {
          const bool rs = co_await restart_check(I, false);
          if (rs || outer == 1) brk = true;
        }
        if (!brk && O.use_duality_gap_restart && O.duality_gap_restart_freq > 0 &&
            S.iter % O.duality_gap_restart_freq == 0) {
          const bool rs = co_await restart_check(I, I.dgap_flag);
          if (rs || outer == 1) brk = true;
        }
        if (brk) {
          restart = true;
          break;
        }
        S.active = 1;
        continue;
      }
    }
    co_await omega_update(I, xds_, yds_);
  }
  I.exit_code = PDCS_EXIT_MAX_ITER;
}

int BatchSolver::prepare() {
  int rc = validate_batch();
  if (rc != PDCS_OK) return rc;
  const double t0 = now_s();
  merge();
  if (O.verbose) std::printf("[pdcs_b200 setup] %-28s %8.3f ms\n", "merge (host)", 1e3 * (now_s() - t0));
  rc = validate();
  if (rc != PDCS_OK) return rc;
  inst_of_y_ = h_iy_.data();
  inst_of_x_ = h_ix_.data();
  setup();
  setup_batch();
  phase("batch constants");
  setup_compaction();
  setup_tiles();
  phase("compaction, tiles");
  setup_act_lists();
  phase("active lists");
  setup_fused();
  phase("fused tiles");
  // the merged matrix lives on the device now (its row pointers stay for the adjoint's scatter)
  std::vector<int64_t>().swap(h_src_);
  if (!O.differentiable) std::vector<int32_t>().swap(h_rp_);
  if (O.differentiable) {
    xs_raw_ = A.alloc<double>(n_);
    ys_raw_ = A.alloc<double>(m_);
    XA_ = XI;
    XA_.S = nullptr;
    XA_.lo = bl_raw_;
    XA_.hi = bu_raw_;
    XA_.rho_ws = nullptr;
    XA_.soc_ws = nullptr;
    YA_ = YI;
    YA_.S = nullptr;
    YA_.rho_ws = nullptr;
    YA_.soc_ws = nullptr;
  }
  P.G_rowptr = nullptr;
  P.G_colind = nullptr;
  P.G_val = nullptr;
  setup_time_ = now_s() - t0;
  prepared_ = true;
  return PDCS_OK;
}

// iterates to the cold start, warm starts of the exponential-cone roots cleared,
// fresh per-instance control state
void BatchSolver::reset_state() {
  for (double* v : {x, xl, xm, xbest}) PDCS_CUDA(cudaMemsetAsync(v, 0, sizeof(double) * n_, s_));
  for (double* v : {y, yl, ym, ybest}) PDCS_CUDA(cudaMemsetAsync(v, 0, sizeof(double) * m_, s_));
  const int64_t nxe = XI.exp_count + XI.dexp_count, nye = YI.exp_count + YI.dexp_count;
  if (nxe) PDCS_CUDA(cudaMemsetAsync(XI.rho_ws, 0xff, sizeof(double) * nxe, s_));
  if (nye) PDCS_CUDA(cudaMemsetAsync(YI.rho_ws, 0xff, sizeof(double) * nye, s_));
  if (XI.nwc) PDCS_CUDA(cudaMemsetAsync(XI.soc_ws, 0xff, sizeof(double) * XI.nwc, s_));
  if (YI.nwc) PDCS_CUDA(cudaMemsetAsync(YI.soc_ws, 0xff, sizeof(double) * YI.nwc, s_));
  PDCS_CUDA(cudaMemsetAsync(live_cnt_, 0, 4 * sizeof(int32_t), s_));
  PDCS_CUDA(cudaMemsetAsync(done_ctas_, 0, sizeof(uint32_t), s_));
  act_set_.clear();
  inst_.clear();
  inst_.resize(K_);
  for (int64_t k = 0; k < K_; ++k) {
    Inst& I = inst_[k];
    const InstConst& c = consts_[k];
    I.k = k;
    I.hNrm1 = c.hNrm1;
    I.hNrmInf = c.hNrmInf;
    I.cNrm1 = c.cNrm1;
    I.cNrmInf = c.cNrmInf;
    I.ginf = c.ginf;
    I.omega0 = c.omega0;
  }
  kernels_ = graphs_ = probes_ = rounds_ = tail_rounds_ = 0;
  t_iter_ = 0.0;
  iter_s_ = 0.0;
  dev_ms_ = 0.0;
  for (int t = 0; t < 2; ++t) {
    gev_n_[t] = 0;
    for (double& v : gev_ms_[t]) v = 0.0;
  }
  for (int t = 0; t < 16; ++t) {
    svc_s_[t] = 0.0;
    svc_groups_[t] = svc_insts_[t] = 0;
  }
}

int BatchSolver::solve(pdcs_result* res, pdcs_batch_info* info, int64_t attempt_limit) {
  if (!prepared_) return PDCS_ERR_INVALID;
  const int64_t limit0 = O.attempt_limit;
  if (attempt_limit > 0) O.attempt_limit = attempt_limit;
  reset_state();
  t_start_ = now_s();
  schedule();
  O.attempt_limit = limit0;
  if (O.verbose) {
    static const char* names[] = {"none", "iterate", "converge", "probe", "mnorm", "seg",
                                  "lin",  "spmv",    "reflect",  "bsearch"};
    std::printf("[pdcs_b200 batch] schedule %.3f s: iteration rounds %.3f s", now_s() - t_start_, iter_s_);
    for (int t = 0; t < 10; ++t)
      if (svc_groups_[t])
        std::printf(", %s %lld groups / %lld requests %.3f s", names[t], (long long)svc_groups_[t],
                    (long long)svc_insts_[t], svc_s_[t]);
    std::printf("\n[pdcs_b200 batch] iteration graphs: device time %.3f s\n", 1e-3 * dev_ms_);
    static const char* kn[6] = {"G'y", "primal", "Gx", "dual", "control", "reflect"};
    for (int t = 0; t < 2; ++t)
      if (gev_n_[t]) {
        std::printf("[pdcs_b200 batch] %s graph, last attempt of %lld rounds, mean us:", t ? "tail" : "full",
                    (long long)gev_n_[t]);
        for (int i = 0; i < 6; ++i) std::printf(" %s %.1f", kn[i], 1e3 * gev_ms_[t][i] / gev_n_[t]);
        std::printf("\n");
      }
  }
  PDCS_CUDA(cudaStreamSynchronize(s_));
  // outputs: unscaled current or averaged iterate per instance, scattered to the callers' buffers
  uint8_t* hpick = stage<uint8_t>(K_);
  for (int64_t k = 0; k < K_; ++k) {
    const Inst& I = inst_[k];
    hpick[k] = (I.exit_code == PDCS_EXIT_OPTIMAL && I.returned_seq == 1) ? 1 : 0;
  }
  PDCS_CUDA(cudaMemcpyAsync(mask_, hpick, K_, cudaMemcpyHostToDevice, s_));
  double* xo = tn[0];
  double* yo = tm[0];
  batch_output_kernel<<<grid_for(n_), kThreads, 0, s_>>>(xo, x, xm, Dr, ix_, mask_, n_);
  batch_output_kernel<<<grid_for(m_), kThreads, 0, s_>>>(yo, y, ym, Dl, iy_, mask_, m_);
  std::vector<double> hx(n_), hy(m_);
  PDCS_CUDA(cudaMemcpyAsync(hx.data(), xo, sizeof(double) * n_, cudaMemcpyDeviceToHost, s_));
  PDCS_CUDA(cudaMemcpyAsync(hy.data(), yo, sizeof(double) * m_, cudaMemcpyDeviceToHost, s_));
  if (O.differentiable) {
    PDCS_CUDA(cudaMemcpyAsync(xs_raw_, xo, sizeof(double) * n_, cudaMemcpyDeviceToDevice, s_));
    PDCS_CUDA(cudaMemcpyAsync(ys_raw_, yo, sizeof(double) * m_, cudaMemcpyDeviceToDevice, s_));
  }
  PDCS_CUDA(cudaStreamSynchronize(s_));
  const double solve_time = now_s() - t_start_;
  int64_t fallbacks = 0;
  for (int64_t k = 0; k < K_; ++k) {
    const Inst& I = inst_[k];
    pdcs_result& R = res[k];
    if (I.needs_single) {
      // resolving fallback (power method + fixed-step PDHG): the single solver
      // replays this instance's trajectory and continues with the fallback
      fallbacks++;
      pdcs_options o1 = O;
      o1.stream = nullptr;
      Solver one(&probs_[k], &o1);
      int r1 = one.run(&R);
      if (r1 != PDCS_OK) return r1;
      if (O.differentiable && R.x && R.y) {  // its solution, for the adjoint
        for (int t = 0; t < kMaxRuns; ++t) {
          std::memcpy(hx.data() + xrun_start_[k * kMaxRuns + t], R.x + xloc_[k * kMaxRuns + t],
                      sizeof(double) * xrun_len_[k * kMaxRuns + t]);
          std::memcpy(hy.data() + yrun_start_[k * kMaxRuns + t], R.y + yloc_[k * kMaxRuns + t],
                      sizeof(double) * yrun_len_[k * kMaxRuns + t]);
        }
        PDCS_CUDA(cudaMemcpy(xs_raw_, hx.data(), sizeof(double) * n_, cudaMemcpyHostToDevice));
        PDCS_CUDA(cudaMemcpy(ys_raw_, hy.data(), sizeof(double) * m_, cudaMemcpyHostToDevice));
      }
      continue;
    }
    for (int t = 0; t < kMaxRuns; ++t) {
      const int64_t L = xrun_len_[k * kMaxRuns + t];
      if (L && R.x)
        std::memcpy(R.x + xloc_[k * kMaxRuns + t], hx.data() + xrun_start_[k * kMaxRuns + t], sizeof(double) * L);
      const int64_t Ly = yrun_len_[k * kMaxRuns + t];
      if (Ly && R.y)
        std::memcpy(R.y + yloc_[k * kMaxRuns + t], hy.data() + yrun_start_[k * kMaxRuns + t], sizeof(double) * Ly);
    }
    const bool mean = hpick[k] != 0;
    const Converge& C = I.ci[mean ? 1 : 0];
    const int ec = I.exit_code;
    R.exit_code = ec;
    R.returned_sequence = mean ? 1 : 0;
    R.pObj = (ec == PDCS_EXIT_OPTIMAL || ec == PDCS_EXIT_MAX_ITER) ? C.pobj : I.pobj;
    R.dObj = (ec == PDCS_EXIT_OPTIMAL || ec == PDCS_EXIT_MAX_ITER) ? C.dobj : I.dobj;
    R.iter = I.S.iter;
    R.restart_used = I.restart_used;
    R.l_inf_rel_primal_res = C.linf_rel_p;
    R.l_inf_rel_dual_res = C.linf_rel_d;
    R.rel_gap = C.rel_gap;
    R.l_2_rel_primal_res = C.l2_rel_p;
    R.l_2_rel_dual_res = C.l2_rel_d;
    R.l_inf_abs_primal_res = C.linf_abs_p;
    R.l_inf_abs_dual_res = C.linf_abs_d;
    R.abs_gap = C.abs_gap;
    R.time = solve_time;
    R.setup_time = setup_time_;
    R.kernel_launches = kernels_;
    R.graph_launches = graphs_;
    R.restart_probes = I.probes;
    R.spmv_lane_nnz_G = lane_G_;
    R.spmv_lane_nnz_Gt = lane_Gt_;
  }
  solved_ = true;
  if (info) {
    info->setup_time = setup_time_;
    info->solve_time = solve_time;
    info->kernel_launches = kernels_;
    info->graph_launches = graphs_;
    info->service_rounds = rounds_;
    info->single_fallbacks = fallbacks;
    info->time_iterations = t_iter_;
    info->spmv_tiled = tiled_ ? 1 : 0;
    info->tail_rounds = (int32_t)tail_rounds_;
  }
  return PDCS_OK;
}

// ---------------------------------------------------------------------------
// Solution-map adjoint (differentiable mode); kernels in pdcs_adjoint.cuh.
// ---------------------------------------------------------------------------
void BatchSolver::scatter_x(const double* merged, double* const* out) const {
  for (int64_t k = 0; k < K_; ++k)
    if (out && out[k])
      for (int t = 0; t < kMaxRuns; ++t)
        std::memcpy(out[k] + xloc_[k * kMaxRuns + t], merged + xrun_start_[k * kMaxRuns + t],
                    sizeof(double) * xrun_len_[k * kMaxRuns + t]);
}

void BatchSolver::scatter_y(const double* merged, double* const* out) const {
  for (int64_t k = 0; k < K_; ++k)
    if (out && out[k])
      for (int t = 0; t < kMaxRuns; ++t)
        std::memcpy(out[k] + yloc_[k * kMaxRuns + t], merged + yrun_start_[k * kMaxRuns + t],
                    sizeof(double) * yrun_len_[k * kMaxRuns + t]);
}

void BatchSolver::set_solution(const double* const* xs, const double* const* ys) {
  std::vector<double> hx(n_, 0.0), hy(m_, 0.0);
  for (int64_t k = 0; k < K_; ++k)
    for (int t = 0; t < kMaxRuns; ++t) {
      if (xs[k])
        std::memcpy(hx.data() + xrun_start_[k * kMaxRuns + t], xs[k] + xloc_[k * kMaxRuns + t],
                    sizeof(double) * xrun_len_[k * kMaxRuns + t]);
      if (ys[k])
        std::memcpy(hy.data() + yrun_start_[k * kMaxRuns + t], ys[k] + yloc_[k * kMaxRuns + t],
                    sizeof(double) * yrun_len_[k * kMaxRuns + t]);
    }
  PDCS_CUDA(cudaMemcpyAsync(xs_raw_, hx.data(), sizeof(double) * n_, cudaMemcpyHostToDevice, s_));
  PDCS_CUDA(cudaMemcpyAsync(ys_raw_, hy.data(), sizeof(double) * m_, cudaMemcpyHostToDevice, s_));
  PDCS_CUDA(cudaStreamSynchronize(s_));
  solved_ = true;
}

void BatchSolver::setup_adjoint(int mr) {
  if (adj_.mr >= mr) return;
  const int64_t N = n_ + m_;
  adj_.mr = mr;
  adj_.V = A.alloc<double>((size_t)(mr + 1) * N);
  if (!adj_.g) {
    adj_.g = A.alloc<double>(N);
    adj_.u = A.alloc<double>(N);
    adj_.Au = A.alloc<double>(N);
    for (double** v : {&adj_.a, &adj_.xp, &adj_.tt, &adj_.tq, &adj_.tr, &adj_.ttr, &adj_.Tx}) *v = A.alloc<double>(n_);
    for (double** v : {&adj_.b, &adj_.tw, &adj_.tsw, &adj_.ts, &adj_.Sy}) *v = A.alloc<double>(m_);
    adj_.dG = A.alloc<double>(nnz_);
    adj_.mask = A.alloc<uint8_t>(K_);
  }
  for (double** v : {&adj_.coef, &adj_.dots1, &adj_.dots2, &adj_.dotsn}) *v = A.alloc<double>((size_t)K_ * (mr + 1));
  adj_.H = A.alloc<double>((size_t)K_ * (mr + 1) * mr);
  adj_.cs = A.alloc<double>((size_t)K_ * mr);
  adj_.sn = A.alloc<double>((size_t)K_ * mr);
  adj_.gam = A.alloc<double>((size_t)K_ * (mr + 1));
  if (!adj_.dpart) {
    adj_.dpart = A.alloc<double>((size_t)K_ * kAdjSplit * 8);
    adj_.beta0 = A.alloc<double>(K_);
    adj_.res = A.alloc<double>(K_);
    adj_.jk = A.alloc<int32_t>(K_);
    adj_.iters = A.alloc<int64_t>(K_);
    adj_.run = A.alloc<uint8_t>(K_);
  }
}

// out = (I - M') u on the masked instances
void BatchSolver::apply_AT(const double* u, double* out, const uint8_t* mask) {
  auto cta = [](int64_t v) { return (int)std::max<int64_t>(1, std::min<int64_t>(v, 148 * 8)); };
  const int wy = YA_.nwc ? cta((YA_.nwc + kWarps - 1) / kWarps) : 0;
  const int wx = XA_.nwc ? cta((XA_.nwc + kWarps - 1) / kWarps) : 0;
  jac_kernel<<<std::max(1, YA_.ctaA + wy + YA_.ctaC), kThreads, 0, s_>>>(YA_, wy, adj_.b, u + n_, adj_.tw, iy_, mask);
  adj_mul_kernel<<<grid_for(m_), kThreads, 0, s_>>>(m_, adj_.Sy, adj_.tw, adj_.tsw);
  spmv_masked(Gtraw_, adj_.tsw, adj_.tt, mask);
  adj_q_kernel<<<grid_for(n_), kThreads, 0, s_>>>(n_, ix_, mask, u, adj_.tt, adj_.tq);
  jac_kernel<<<std::max(1, XA_.ctaA + wx + XA_.ctaC), kThreads, 0, s_>>>(XA_, wx, adj_.a, adj_.tq, adj_.tr, ix_, mask);
  adj_mul_kernel<<<grid_for(n_), kThreads, 0, s_>>>(n_, adj_.Tx, adj_.tr, adj_.ttr);
  spmv_masked(Graw_, adj_.ttr, adj_.ts, mask);
  adj_finish_kernel<<<grid_for(n_ + m_), kThreads, 0, s_>>>(n_, m_, ix_, iy_, mask, u, adj_.tr, adj_.tt, adj_.tw,
                                                           adj_.ts, out);
  kernels_ += 6;
}

int BatchSolver::grad(const double* const* dldx, const double* const* dldy, double* const* dc, double* const* dh,
                      double* const* dG, double* const* dl, double* const* du, const pdcs_grad_options& go,
                      pdcs_grad_info* info) {
  if (!O.differentiable || !solved_) return PDCS_ERR_INVALID;
  const double t0 = now_s();
  const int mr = std::max(2, std::min(go.restart > 0 ? go.restart : 100, 200));
  const double tol = go.rel_tol > 0 ? go.rel_tol : 1e-10;
  const int64_t maxit = go.max_iter > 0 ? go.max_iter : 5000;
  setup_adjoint(mr);
  const int64_t N = n_ + m_, K = K_;
  const int ld = adj_.mr + 1;
  // block-constant Pock-Chambolle steps: T = 0.9 / column sums, S = 0.9 / row sums of |G|
  row_absstat_kernel<true><<<warp_grid(m_), kThreads, 0, s_>>>(m_, Graw_.rp, Graw_.v, nullptr, adj_.Sy);
  row_absstat_kernel<true><<<warp_grid(n_), kThreads, 0, s_>>>(n_, Gtraw_.rp, Gtraw_.v, nullptr, adj_.Tx);
  adj_steps_kernel<<<grid_for(m_), kThreads, 0, s_>>>(m_, adj_.Sy);
  adj_steps_kernel<<<grid_for(n_), kThreads, 0, s_>>>(n_, adj_.Tx);
  adj_block_min_kernel<<<grid_for(std::max(n_, m_)), kThreads, 0, s_>>>(XA_, adj_.Tx);
  adj_block_min_kernel<<<grid_for(std::max(n_, m_)), kThreads, 0, s_>>>(YA_, adj_.Sy);
  // projection points a = x + T (G'y - c), b = y - S (G (2 P_X(a) - x) - h)
  spmv(Gtraw_, ys_raw_, adj_.tt);
  adj_point_kernel<<<grid_for(n_), kThreads, 0, s_>>>(n_, adj_.Tx, xs_raw_, adj_.tt, c_raw, 1.0, adj_.a);
  OpAxpyProj px{adj_.a, adj_.a, 0.0, adj_.xp, nullptr, nullptr};
  update_project(px, XA_, part_a);
  axpby_kernel<<<grid_for(n_), kThreads, 0, s_>>>(adj_.tq, 2.0, adj_.xp, -1.0, xs_raw_, n_);
  spmv(Graw_, adj_.tq, adj_.ts);
  adj_point_kernel<<<grid_for(m_), kThreads, 0, s_>>>(m_, adj_.Sy, ys_raw_, adj_.ts, h_raw, -1.0, adj_.b);
  kernels_ += 9;
  // right-hand side g = (dL/dx*, dL/dy*) in the merged layout
  {
    std::vector<double> hg(N, 0.0);
    for (int64_t k = 0; k < K; ++k)
      for (int t = 0; t < kMaxRuns; ++t) {
        if (dldx && dldx[k])
          std::memcpy(hg.data() + xrun_start_[k * kMaxRuns + t], dldx[k] + xloc_[k * kMaxRuns + t],
                      sizeof(double) * xrun_len_[k * kMaxRuns + t]);
        if (dldy && dldy[k])
          std::memcpy(hg.data() + n_ + yrun_start_[k * kMaxRuns + t], dldy[k] + yloc_[k * kMaxRuns + t],
                      sizeof(double) * yrun_len_[k * kMaxRuns + t]);
      }
    PDCS_CUDA(cudaMemcpyAsync(adj_.g, hg.data(), sizeof(double) * N, cudaMemcpyHostToDevice, s_));
    PDCS_CUDA(cudaMemsetAsync(adj_.u, 0, sizeof(double) * N, s_));
    PDCS_CUDA(cudaStreamSynchronize(s_));
  }
  // CTAs per instance in the dot products: enough CTAs to fill the GPU (a CTA per instance
  // when the batch is large), capped at kAdjSplit
  const int split = (int)std::max<int64_t>(1, std::min<int64_t>(kAdjSplit, (148 * 8 + K - 1) / K));
  const int dgrid = (int)std::max<int64_t>(1, std::min<int64_t>(K * split, 148 * 8));
  // per-instance dot products <V_p, w>, p < np, into out (device; no synchronisation)
  auto dots = [&](const uint8_t* mask, const double* V, int np, const double* w, double* out) {
    for (int q = 0; q < np; q += 8) {
      const int c = std::min(8, np - q);
      adj_dots_kernel<<<dgrid, kThreads, 0, s_>>>(K, split, mask, rx_, ry_, n_, V, N, q, c, w, adj_.dpart);
      adj_dots_reduce_kernel<<<grid_for(K * c), kThreads, 0, s_>>>(K, split, mask, q, c, adj_.dpart, out, ld);
      kernels_ += 2;
    }
  };
  auto fetch = [&](const double* dev) {
    double* h = stage<double>((size_t)K * ld);
    PDCS_CUDA(cudaMemcpyAsync(h, dev, sizeof(double) * K * ld, cudaMemcpyDeviceToHost, s_));
    return h;
  };
  auto upload_mask8 = [&](const std::vector<uint8_t>& act) {
    uint8_t* h = stage<uint8_t>(K);
    std::memcpy(h, act.data(), K);
    PDCS_CUDA(cudaMemcpyAsync(adj_.mask, h, K, cudaMemcpyHostToDevice, s_));
  };
  auto any = [](const std::vector<uint8_t>& v) { return std::any_of(v.begin(), v.end(), [](uint8_t b) { return b; }); };
  std::vector<double> beta0(K), res(K, 0.0);
  std::vector<int64_t> iters(K, 0);
  std::vector<uint8_t> conv(K, 0);
  {
    dots(nullptr, adj_.g, 1, adj_.g, adj_.dotsn);
    const double* h = fetch(adj_.dotsn);
    PDCS_CUDA(cudaStreamSynchronize(s_));
    for (int64_t k = 0; k < K; ++k) {
      beta0[k] = std::sqrt(h[k * ld]);
      conv[k] = beta0[k] > 0 ? 0 : 1;
    }
    double* hb = stage<double>(K);
    for (int64_t k = 0; k < K; ++k) hb[k] = beta0[k] > 0 ? beta0[k] : 1.0;
    PDCS_CUDA(cudaMemcpyAsync(adj_.beta0, hb, sizeof(double) * K, cudaMemcpyHostToDevice, s_));
    PDCS_CUDA(cudaMemsetAsync(adj_.iters, 0, sizeof(int64_t) * K, s_));
  }
  // restarted GMRES: one Arnoldi process per instance, all instances per launch;
  // classical Gram-Schmidt twice, the Hessenberg column, Givens rotations and the
  // back substitution on the device (adj_givens_kernel, adj_backsub_kernel), so a
  // step needs no host round trip; the host looks at the mask every kCheck steps
  constexpr int kCheck = 8;
  const int kg = (int)std::max<int64_t>(1, std::min<int64_t>((K + kThreads - 1) / kThreads, 148));
  double* V = adj_.V;
  int64_t total_it = 0;
  bool first = true;
  while (total_it < maxit) {
    std::vector<uint8_t> run(K);
    for (int64_t k = 0; k < K; ++k) run[k] = !conv[k];
    if (!any(run)) break;
    upload_mask8(run);
    if (first) {
      copy(V, adj_.g, N);
    } else {  // V_0 = g - A u
      apply_AT(adj_.u, adj_.Au, adj_.mask);
      axpby_kernel<<<grid_for(N), kThreads, 0, s_>>>(V, 1.0, adj_.g, -1.0, adj_.Au, N);
      kernels_++;
    }
    first = false;
    dots(adj_.mask, V, 1, V, adj_.dotsn);
    const double* hb = fetch(adj_.dotsn);
    adj_normalize_kernel<<<grid_for(N), kThreads, 0, s_>>>(N, n_, ix_, iy_, adj_.mask, adj_.dotsn, ld, V);
    kernels_++;
    PDCS_CUDA(cudaStreamSynchronize(s_));
    double* hg = stage<double>(K);  // gamma = (beta, 0, ..., 0) per instance
    for (int64_t k = 0; k < K; ++k) {
      hg[k] = 0.0;
      if (!run[k]) continue;
      const double beta = std::sqrt(hb[k * ld]);
      res[k] = beta / beta0[k];
      if (beta <= tol * beta0[k]) {
        conv[k] = 1;
        run[k] = 0;
        continue;
      }
      hg[k] = beta;
    }
    if (!any(run)) break;
    {  // the cycle's instances: the Arnoldi mask and the back substitution's
      PDCS_CUDA(cudaMemsetAsync(adj_.gam, 0, sizeof(double) * K * (mr + 1), s_));
      PDCS_CUDA(cudaMemcpy2DAsync(adj_.gam, sizeof(double) * (mr + 1), hg, sizeof(double), sizeof(double), K,
                                  cudaMemcpyHostToDevice, s_));
      upload_mask8(run);
      PDCS_CUDA(cudaMemcpyAsync(adj_.run, adj_.mask, K, cudaMemcpyDeviceToDevice, s_));
      PDCS_CUDA(cudaMemsetAsync(adj_.jk, 0, sizeof(int32_t) * K, s_));
    }
    for (int j = 0; j < mr && total_it < maxit; ++j) {
      if (j > 0 && j % kCheck == 0) {  // every instance done extending its basis: end the cycle
        uint8_t* hm = stage<uint8_t>(K);
        PDCS_CUDA(cudaMemcpyAsync(hm, adj_.mask, K, cudaMemcpyDeviceToHost, s_));
        PDCS_CUDA(cudaStreamSynchronize(s_));
        if (!std::any_of(hm, hm + K, [](uint8_t v) { return v != 0; })) break;
      }
      double* W = V + (size_t)(j + 1) * N;
      apply_AT(V + (size_t)j * N, W, adj_.mask);
      dots(adj_.mask, V, j + 1, W, adj_.dots1);
      adj_combine_kernel<<<grid_for(N), kThreads, 0, s_>>>(N, n_, ix_, iy_, adj_.mask, V, N, j + 1, adj_.dots1, ld,
                                                          -1.0, W);
      dots(adj_.mask, V, j + 1, W, adj_.dots2);
      adj_combine_kernel<<<grid_for(N), kThreads, 0, s_>>>(N, n_, ix_, iy_, adj_.mask, V, N, j + 1, adj_.dots2, ld,
                                                          -1.0, W);
      dots(adj_.mask, W, 1, W, adj_.dotsn);
      adj_normalize_kernel<<<grid_for(N), kThreads, 0, s_>>>(N, n_, ix_, iy_, adj_.mask, adj_.dotsn, ld, W);
      adj_givens_kernel<<<kg, kThreads, 0, s_>>>(K, j, mr, ld, adj_.mask, adj_.dots1, adj_.dots2, adj_.dotsn, adj_.H,
                                                 adj_.cs, adj_.sn, adj_.gam, adj_.beta0, tol, adj_.jk, adj_.iters,
                                                 adj_.res);
      kernels_ += 4;
      total_it++;
    }
    // u += V y, y = H^{-1} gamma (back substitution per instance on the device)
    adj_backsub_kernel<<<kg, kThreads, 0, s_>>>(K, mr, ld, adj_.run, adj_.jk, adj_.H, adj_.gam, adj_.coef);
    kernels_++;
    int32_t* hj = stage<int32_t>(K);
    PDCS_CUDA(cudaMemcpyAsync(hj, adj_.jk, sizeof(int32_t) * K, cudaMemcpyDeviceToHost, s_));
    PDCS_CUDA(cudaStreamSynchronize(s_));
    int jmax = 0;
    for (int64_t k = 0; k < K; ++k)
      if (run[k]) jmax = std::max(jmax, (int)hj[k]);
    if (jmax > 0) {
      adj_combine_kernel<<<grid_for(N), kThreads, 0, s_>>>(N, n_, ix_, iy_, adj_.run, V, N, jmax, adj_.coef, ld, 1.0,
                                                          adj_.u);
      kernels_++;
    }
  }
  {
    int64_t* hi = stage<int64_t>(K);
    PDCS_CUDA(cudaMemcpyAsync(hi, adj_.iters, sizeof(int64_t) * K, cudaMemcpyDeviceToHost, s_));
    PDCS_CUDA(cudaStreamSynchronize(s_));
    for (int64_t k = 0; k < K; ++k) iters[k] = hi[k];
  }
  // true relative residuals |g - A u| / |g|
  {
    std::vector<uint8_t> all(K, 1);
    upload_mask8(all);
    apply_AT(adj_.u, adj_.Au, adj_.mask);
    axpby_kernel<<<grid_for(N), kThreads, 0, s_>>>(adj_.Au, 1.0, adj_.g, -1.0, adj_.Au, N);
    kernels_++;
    dots(nullptr, adj_.Au, 1, adj_.Au, adj_.dotsn);
    const double* h = fetch(adj_.dotsn);
    PDCS_CUDA(cudaStreamSynchronize(s_));
    for (int64_t k = 0; k < K; ++k) res[k] = beta0[k] > 0 ? std::sqrt(h[k * ld]) / beta0[k] : 0.0;
  }
  // parameter gradients: w = D_K u_y, t = G' (S w), q = u_x - 2 t, r = D_X q
  {
    std::vector<uint8_t> all(K, 1);
    upload_mask8(all);
    apply_AT(adj_.u, adj_.Au, adj_.mask);  // leaves w (tw), q (tq), r (tr) of u in the work vectors
    // outputs in the Krylov basis storage (no longer needed; (mr + 1) N >= 3 N entries):
    // dh over y at V, dc over x then dl, du over the box part at V + N
    double* dhv = adj_.V;
    double* dcv = adj_.V + N;
    double* dlv = dcv + n_;
    double* duv = dcv + n_ + nb_;
    adj_dc_kernel<<<grid_for(n_), kThreads, 0, s_>>>(n_, nb_, adj_.Tx, adj_.tr, adj_.tq, adj_.a, bl_raw_, bu_raw_,
                                                     dcv, dlv, duv);
    adj_mul_kernel<<<grid_for(m_), kThreads, 0, s_>>>(m_, adj_.Sy, adj_.tw, dhv);
    adj_dG_kernel<<<warp_grid(m_), kThreads, 0, s_>>>(m_, Graw_.rp, Graw_.ci, adj_.Tx, adj_.Sy, ys_raw_, adj_.tw,
                                                      xs_raw_, adj_.tr, adj_.dG);
    kernels_ += 3;
    std::vector<double> hdc(n_ + 2 * nb_), hdh(m_), hdG(dG ? nnz_ : 0);
    PDCS_CUDA(cudaMemcpyAsync(hdc.data(), dcv, sizeof(double) * (n_ + 2 * nb_), cudaMemcpyDeviceToHost, s_));
    PDCS_CUDA(cudaMemcpyAsync(hdh.data(), dhv, sizeof(double) * m_, cudaMemcpyDeviceToHost, s_));
    if (dG) PDCS_CUDA(cudaMemcpyAsync(hdG.data(), adj_.dG, sizeof(double) * nnz_, cudaMemcpyDeviceToHost, s_));
    PDCS_CUDA(cudaStreamSynchronize(s_));
    scatter_x(hdc.data(), dc);
    scatter_y(hdh.data(), dh);
    for (int64_t k = 0; k < K; ++k) {
      const int64_t b0 = xrun_start_[k * kMaxRuns], nb = xrun_len_[k * kMaxRuns];
      if (dl && dl[k]) std::memcpy(dl[k], hdc.data() + n_ + b0, sizeof(double) * nb);
      if (du && du[k]) std::memcpy(du[k], hdc.data() + n_ + nb_ + b0, sizeof(double) * nb);
      if (dG && dG[k]) {  // merged entries keep each row's order: copy row by row
        const pdcs_problem& q = probs_[k];
        for (int64_t i = 0; i < q.m; ++i)
          std::memcpy(dG[k] + q.G_rowptr[i], hdG.data() + h_rp_[merged_row(k, i)],
                      sizeof(double) * (q.G_rowptr[i + 1] - q.G_rowptr[i]));
      }
    }
  }
  const double t1 = now_s();
  if (info)
    for (int64_t k = 0; k < K; ++k) {
      info[k].iterations = iters[k];
      info[k].residual = res[k];
      info[k].time = t1 - t0;
      info[k].converged = res[k] <= std::max(10 * tol, 1e-8) ? 1 : 0;
    }
  return PDCS_OK;
}

}  // namespace pdcs
