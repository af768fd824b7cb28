/*
 * pdcs.h -- C ABI of the B200-native PDHG conic solver (libpdcs_b200.so).
 *
 * Problem form (PDCS README.md:9-15):
 *     min c'x  s.t.  Gx - h in K_d,  bl <= x[0:nb] <= bu,  x[nb:] in K_p
 *   x = [box (nb) | SOC blocks (soc_x) | RSOC blocks (rsoc_x) | exp (3 each) | dual-exp (3 each)]
 *   y = [zero (mGzero) | nonneg (mGnonnegative) | SOC (socG) | RSOC (rsocG) | exp x3 | dual-exp x3]
 *   (layout of src/pdcs_gpu/rpdhg_alg_gpu_gen.jl:60-120).
 *
 * Ownership: the caller owns every input and output buffer; the library owns
 * its device workspace for the duration of one call.  Errors are returned as
 * negative status codes (the reference's Julia API throws instead:
 * rpdhg_alg_gpu_gen.jl:1331-1375, :84, :94); solve outcomes are the
 * reference's exit codes (def_struct.jl:735-745, termination.jl:188-258).
 * Threading: each call is self-contained and runs on one stream of the
 * current CUDA device; independent calls may run concurrently on different
 * streams.
 */
#ifndef PDCS_B200_H
#define PDCS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (negative: the call did not run) ---------------------- */
#define PDCS_OK 0
#define PDCS_ERR_INVALID (-1)        /* null pointer / inconsistent sizes      */
#define PDCS_ERR_CUDA (-2)           /* a CUDA runtime call failed             */
#define PDCS_ERR_M_MISMATCH (-3)     /* m != mGzero+mGnonneg+sum(socG)+sum(rsocG)+3(expG+dual_expG) */
#define PDCS_ERR_SOC_DIM (-4)        /* an SOC block has dimension < 2         */
#define PDCS_ERR_RSOC_DIM (-5)       /* an RSOC block has dimension < 3        */
#define PDCS_ERR_BOUNDS (-6)         /* some bl[j] > bu[j]                     */
#define PDCS_ERR_N_MISMATCH (-7)     /* cone blocks of x exceed n              */
#define PDCS_ERR_NO_DEVICE (-8)      /* no CUDA device                         */
#define PDCS_ERR_UNSUPPORTED (-9)    /* option combination not implemented     */
#define PDCS_ERR_NOALLOC_LIMIT (-10) /* problem exceeds the fixed scratch of pdcs_spmv_csr_noalloc */

/* ---- solver exit codes (pdcs_result.exit_code), as the reference --------- */
#define PDCS_EXIT_OPTIMAL 0
#define PDCS_EXIT_MAX_ITER 1
#define PDCS_EXIT_PRIMAL_INFEASIBLE_LOW_ACC 2
#define PDCS_EXIT_PRIMAL_INFEASIBLE_HIGH_ACC 3
#define PDCS_EXIT_DUAL_INFEASIBLE_LOW_ACC 4
#define PDCS_EXIT_DUAL_INFEASIBLE_HIGH_ACC 5
#define PDCS_EXIT_TIME_LIMIT 6
#define PDCS_EXIT_CONTINUE 7
#define PDCS_EXIT_NUMERICAL_NAN 8
#define PDCS_EXIT_NUMERICAL_INF 9
#define PDCS_EXIT_ATTEMPT_LIMIT 10   /* stopped by pdcs_options.attempt_limit (benchmark sampling) */

/* ---- projection codes for pdcs_block_proj (def_rpdhg_gen.jl:265-279, 598-616) */
/*  0/1 free, 2 zero, 3/4 nonneg, 5/7/20/21 SOC, 6/22 S-scaled SOC, 8/10/23/24 RSOC,
 *  9/25 S-scaled RSOC, 11/16/28 dual-exp, 12/29 S o K_exp^*, 13/14/26 exp,
 *  15/27 S o K_exp, 17/18/19 box clamp [bl, bu].                                  */

typedef struct {
  int64_t n, m, nb, nnz;
  const int32_t* G_rowptr; /* m + 1, 0-based CSR of G (m x n)   */
  const int32_t* G_colind; /* nnz                               */
  const double* G_val;     /* nnz                               */
  const double* c;         /* n                                 */
  const double* h;         /* m                                 */
  const double* bl;        /* nb, may hold -INFINITY            */
  const double* bu;        /* nb, may hold +INFINITY            */
  int64_t mGzero, mGnonnegative;
  const int64_t* socG;  int64_t n_socG;
  const int64_t* rsocG; int64_t n_rsocG;
  int64_t expG, dual_expG;
  const int64_t* soc_x;  int64_t n_soc_x;
  const int64_t* rsoc_x; int64_t n_rsoc_x;
  int64_t exp_x, dual_exp_x;
  int32_t on_device;       /* 1: G_*, c, h, bl, bu are device pointers of the current device */
  int32_t reserved;
} pdcs_problem;

/* Mirrors the keyword arguments of rpdhg_gpu_solve (rpdhg_alg_gpu_gen.jl:1219-1268). */
typedef struct {
  int32_t rescaling_method;      /* 0 none, 1 ruiz, 2 pock_chambolle, 3 ruiz_pock_chambolle (default) */
  int32_t use_preconditioner;    /* 1 */
  int32_t use_adaptive_restart;  /* 1 */
  int32_t use_adaptive_step_size_weight; /* 1 */
  int32_t use_aggressive;        /* 1 */
  int32_t use_accelerated;       /* 0 */
  int32_t use_resolving;         /* 1 */
  int32_t warm_start;            /* 0 */
  const double* primal_sol;      /* n (host), used when warm_start */
  const double* dual_sol;        /* m (host), used when warm_start */
  int64_t max_outer_iter;        /* 10000  */
  int64_t max_inner_iter;        /* 500000 */
  double abs_tol, rel_tol;       /* 1e-6   */
  double eps_primal_infeasible_low_acc, eps_dual_infeasible_low_acc;   /* 1e-12 */
  double eps_primal_infeasible_high_acc, eps_dual_infeasible_high_acc; /* 1e-16 */
  int64_t print_freq;            /* 2000 */
  int64_t check_terminate_freq;  /* 2000 */
  int32_t verbose;               /* 0 */
  int32_t use_kkt_restart;       /* 0 */
  double time_limit;             /* seconds; <= 0 means none */
  int64_t kkt_restart_freq;      /* 2000 */
  int32_t use_duality_gap_restart; /* 1 */
  int32_t precision;             /* 0: FP64 throughout (the reference's arithmetic); 1: FP32 matrices and
                                    iterate deltas between FP64 anchors (FP64 projections, averages,
                                    termination checks) */
  int64_t duality_gap_restart_freq; /* 2000 */
  int64_t attempt_limit;         /* > 0: stop after this many PDHG attempts (sampling) */
  void* stream;                  /* cudaStream_t to run on; NULL = an internal stream */
  int32_t attempts_per_graph;    /* PDHG attempts captured per CUDA graph (default 32) */
  int32_t force_resolving;       /* test hook: enter the resolving fallback at the first outer iteration */
  int32_t spmv_lane_nnz;         /* SpMV schedule, nonzeros per lane of a row's lane group (power of two,
                                    1..16); 0 (default) = autotuned per matrix at setup for matrices of
                                    2^20 or more nonzeros, 4 below */
  int32_t differentiable;        /* keep the unscaled data the solution-map adjoint (pdcs_batch_grad) needs */
  int32_t spmv_tiles;            /* batched solver's iteration SpMVs: 0 (default) instance tiles -- each CTA
                                    stages one instance's column segment in shared memory, 16-bit local
                                    column indices -- when every instance has at most 65535 variables and
                                    65535 constraint rows; > 0 the same with at most this many nonzeros
                                    per tile (default 65536); -1 the binned row schedule (spmv_lane_nnz).
                                    Rounds with few nonzeros left iterating run the binned schedule */
  int32_t reserved;
} pdcs_options;

typedef struct {
  double* x;                 /* out (host, n) or NULL: recovered primal solution */
  double* y;                 /* out (host, m) or NULL: recovered dual solution   */
  double* x_device;          /* out (device, n) or NULL */
  double* y_device;          /* out (device, m) or NULL */
  int32_t exit_code;         /* PDCS_EXIT_*            */
  int32_t returned_sequence; /* 0 current iterate, 1 averaged iterate */
  double pObj, dObj;
  int64_t iter;              /* PDHG attempts (info.iter) */
  int64_t restart_used;
  double time;               /* main-loop seconds (info.time; excludes preprocessing) */
  double setup_time;         /* upload + preconditioning seconds */
  double l_inf_rel_primal_res, l_inf_rel_dual_res, rel_gap;
  double l_2_rel_primal_res, l_2_rel_dual_res;
  double l_inf_abs_primal_res, l_inf_abs_dual_res, abs_gap;
  int64_t kernel_launches;   /* kernels launched by the library in the main loop */
  int64_t graph_launches;
  double time_iterations;    /* seconds in PDHG attempts (CUDA graphs)            */
  double time_exit_checks;   /* seconds in termination checks (every check_terminate_freq) */
  double time_restarts;      /* seconds in restart thresholds / restart checks    */
  int64_t restart_probes;    /* projections probes of the restart binary searches */
  int32_t spmv_lane_nnz_G;   /* SpMV schedules used for G and G' (nonzeros per lane) */
  int32_t spmv_lane_nnz_Gt;
} pdcs_result;

/* Fills *opts with the reference's defaults. */
int pdcs_default_options(pdcs_options* opts);

/* Solve one conic program.  Replaces rpdhg_gpu_solve / rpdhg_gpu_solve_input_gpu_data
 * (rpdhg_alg_gpu_gen.jl:1219, :387) and the main loop they run
 * (rpdhg_alg_gpu_gen_scaling.jl:770-895). */
int pdcs_solve(const pdcs_problem* prob, const pdcs_options* opts, pdcs_result* res);

/* Totals of one batched solve. */
typedef struct {
  double setup_time;        /* merge + upload + preconditioning seconds */
  double solve_time;        /* scheduler seconds (all instances, incl. the output gather) */
  double time_iterations;   /* seconds in shared CUDA graphs of PDHG attempts */
  int64_t kernel_launches;  /* kernels launched by the batched scheduler */
  int64_t graph_launches;
  int64_t service_rounds;   /* batched checkpoint operations (exit checks, restart probes, copies) */
  int64_t single_fallbacks; /* instances re-solved alone for the resolving fallback */
  int32_t spmv_tiled;       /* 1: the iteration graph ran the instance-tiled SpMV, 0: the binned one */
  int32_t tail_rounds;      /* iteration rounds run by the tail kernel (a CTA per remaining instance) */
} pdcs_batch_info;

/* Solve `count` independent conic programs together.  No counterpart in the
 * reference, whose rpdhg_gpu_solve takes one program; each instance here
 * follows that solver's algorithm with its own step sizes, primal weight,
 * restarts and termination (results[k] as pdcs_solve would fill it; `time` is
 * the batch's solve time).  Problems must be host data (on_device = 0) whose
 * variables all lie in the box or a cone block (n = nb + sum(soc_x) +
 * sum(rsoc_x) + 3 (exp_x + dual_exp_x)); warm starts are not supported.  An
 * instance that enters the resolving fallback is re-solved alone.  info may
 * be NULL.  Returns PDCS_OK or the first validation error. */
int pdcs_solve_batch(int64_t count, const pdcs_problem* problems, const pdcs_options* opts,
                     pdcs_result* results, pdcs_batch_info* info);

/* A prepared batch: merged, uploaded and preconditioned once, solved any number
 * of times from a cold start (to time solves with the data resident in device
 * memory, or to solve again after a forward pass).  No counterpart in the
 * reference.  The problems' host arrays must stay valid until
 * pdcs_batch_destroy (an instance that enters the resolving fallback is
 * re-solved alone from them).  Not thread-safe: one call at a time per handle. */
typedef struct pdcs_batch pdcs_batch;
int pdcs_batch_create(int64_t count, const pdcs_problem* problems, const pdcs_options* opts, pdcs_batch** out);
/* attempt_limit > 0 overrides the option for this solve. */
int pdcs_batch_solve(pdcs_batch* batch, int64_t attempt_limit, pdcs_result* results, pdcs_batch_info* info);
void pdcs_batch_destroy(pdcs_batch* batch);

/* Solution-map adjoint.  No counterpart in the reference.  The solution
 * (x*, y*) of the unscaled problem is a fixed point of the PDHG map T; with
 * M = dT/dz there, the loss gradient g = (dL/dx*, dL/dy*) pulls back through
 * u = (I - M)^{-T} g (M with Pock-Chambolle diagonal steps, constant on each
 * cone block), solved by restarted GMRES whose operator products use
 * the solver's SpMV kernels and the projection Jacobians (box, nonneg, SOC,
 * RSOC, exponential and dual-exponential cones).  Outputs dL/dc, dL/dh,
 * dL/dG (nonzero values in the problem's own CSR order), dL/dl, dL/du. */
typedef struct {
  double rel_tol;     /* relative residual of the adjoint solve (default 1e-10) */
  int32_t restart;    /* GMRES restart length (default 100, at most 200) */
  int32_t reserved;
  int64_t max_iter;   /* total GMRES iterations (default 5000) */
} pdcs_grad_options;

typedef struct {
  int64_t iterations; /* GMRES iterations of this instance */
  double residual;    /* |g - (I - M)' u| / |g| */
  double time;        /* seconds of the whole adjoint call */
  int32_t converged;
  int32_t reserved;
} pdcs_grad_info;

/* Gradients at the last pdcs_batch_solve of a batch created with
 * options.differentiable = 1.  Every argument array has `count` entries, one
 * per instance (host pointers, each sized like the instance's vector; any
 * array, or entry, may be NULL).  opts may be NULL (defaults). */
int pdcs_batch_grad(pdcs_batch* batch, const double* const* dldx, const double* const* dldy, double* const* dc,
                    double* const* dh, double* const* dG, double* const* dl, double* const* du,
                    const pdcs_grad_options* opts, pdcs_grad_info* info);

/* Gradients of one problem at a given solution (x, y) (host arrays, e.g. from
 * pdcs_solve); the problem's variables must all lie in the box or a cone block. */
int pdcs_grad(const pdcs_problem* prob, const pdcs_options* opts, const double* x, const double* y,
              const double* dldx, const double* dldy, double* dc, double* dh, double* dG, double* dl, double* du,
              const pdcs_grad_options* gopts, pdcs_grad_info* info);

/* Block projections on device memory.  Replaces the projection entry points
 * few_block_proj (cuda/few_block_proj.cu:414-432, bound by gpu_kernel.jl:377-406)
 * and massive/moderate/sufficient_block_proj (cuda/moderate_block_proj.cu:1182,
 * bound by gpu_kernel.jl:114-300), same block table (head_start, ns, blkNum,
 * proj_type) and codes.  Difference: the scaled codes take the cumulative
 * scaling vector S (Dr_product or Dl_product) instead of the derived
 * D_scaled / D_scaled_squared / temp arrays, and every projection is solved
 * to machine precision (no abs_tol / rel_tol).  All pointers are device
 * pointers; S may be NULL for the unscaled codes; bl/bu are used by codes 17-19.
 * stream: cudaStream_t or NULL (legacy default stream).  Returns PDCS_OK or an error. */
int pdcs_block_proj(double* arr, const double* bl, const double* bu, const double* S,
                    const int64_t* head_start, const int64_t* ns, int64_t blkNum,
                    const int64_t* proj_type, void* stream);

/* y = G x for a CSR matrix on device (0-based int32 indices, FP64 values);
 * replaces CUDA.CUSPARSE.mv!('N', ...) of unionPrimalMV! (def_rpdhg_gen.jl:856-858).
 * Applying it to the CSR of G' replaces union_adjoint! (:864-866). */
int pdcs_spmv_csr(int64_t m, int64_t n, int64_t nnz, const int32_t* rowptr, const int32_t* colind,
                  const double* val, const double* x, double* y, void* stream);

/* Same result as pdcs_spmv_csr, without allocating.  No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc -- a host
 * whose device memory is owned by its own pool allocator (Julia's CUDA.jl
 * pool, PyTorch's caching allocator) and must not be bypassed or fragmented,
 * or a latency-critical loop where a driver allocation would stall.  The
 * row-carry scratch is a file-scope device array of 65536 entries, so
 * m + nnz must not exceed 134,217,728 (PDCS_ERR_NOALLOC_LIMIT otherwise);
 * every GPU that loads the library keeps those 768 KiB until the process
 * exits.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress, once per device and context: the cached address is
 * looked up again when the device's context was destroyed and recreated);
 * make that first call before any stream capture.  All calls share the one array: calls that overlap on the
 * GPU (different streams, no ordering) race on it.  Allocates nothing:
 * no cudaMalloc, cudaFree or allocating library routine. */
int pdcs_spmv_csr_noalloc(int64_t m, int64_t n, int64_t nnz, const int32_t* rowptr, const int32_t* colind,
                          const double* val, const double* x, double* y, void* stream);

/* Library version string. */
const char* pdcs_version(void);

#ifdef __cplusplus
}
#endif
#endif /* PDCS_B200_H */
