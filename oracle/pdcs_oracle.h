/*
 * pdcs_oracle.h -- CPU FP64 restatement of the PDCS restarted PDHG conic solver.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA product
 * (pdcs_b200/csrc) is compared against.  Only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline / --impl reference leg may load it.  Nothing in
 * the product links or calls it.
 *
 * Parity status: the reference (Julia + CUDA.jl) cannot run in this
 * environment and ships no golden vectors, so the oracle is pinned by
 * mathematical invariants of the projections (Moreau decomposition,
 * feasibility, complementarity, idempotence, brute-force global search) and by
 * end-to-end KKT criteria, not by reference outputs ("parity unpinned" against
 * the reference binary itself).
 *
 * Problem form (README.md:9-15 of the reference):
 *   min c'x  s.t.  Gx - h in K_d,  l <= x_1 <= u,  x_2 in K_p
 * x = [box (nb) | SOC blocks | RSOC blocks | exp (3 each) | dual-exp (3 each)]
 * y = [zero (mGzero) | nonneg (mGnonneg) | SOC | RSOC | exp x3 | dual-exp x3]
 * (layout: src/pdcs_gpu/rpdhg_alg_gpu_gen.jl:60-120).
 */
#ifndef PDCS_ORACLE_H
#define PDCS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* projection kinds for oracle_project_block */
enum {
  ORC_FREE = 0,
  ORC_ZERO = 1,
  ORC_NONNEG = 2,
  ORC_BOX = 3,    /* clamp to [lo, hi] elementwise */
  ORC_SOC = 4,    /* S o SOC   = {(s, y): ||(S0/S_i) y_i|| <= s}          */
  ORC_RSOC = 5,   /* S o RSOC  = {2 p q >= ||(sqrt(S0 S1)/S_i) z_i||^2}    */
  ORC_EXP = 6,    /* S o K_exp, K_exp = cl{(r,s,t): s>0, s e^{r/s} <= t}   */
  ORC_DEXP = 7    /* S o K_exp^*  (dual exponential cone)                  */
};

typedef struct {
  int64_t n, m, nb, nnz;
  const int64_t* rowptr; /* m+1, 0-based CSR of G (m x n) */
  const int64_t* colind; /* nnz */
  const double* val;     /* nnz */
  const double* c;       /* n */
  const double* h;       /* m */
  const double* bl;      /* nb (may hold -inf) */
  const double* bu;      /* nb (may hold +inf) */
  int64_t mGzero, mGnonneg;
  const int64_t* socG; int64_t n_socG;
  const int64_t* rsocG; int64_t n_rsocG;
  int64_t expG, dual_expG;
  const int64_t* soc_x; int64_t n_soc_x;
  const int64_t* rsoc_x; int64_t n_rsoc_x;
  int64_t exp_x, dual_exp_x;
} oracle_problem;

typedef struct {
  int64_t max_outer_iter;        /* 10000   */
  int64_t max_inner_iter;        /* 500000  */
  double abs_tol, rel_tol;       /* 1e-6    */
  double eps_primal_infeasible_low_acc, eps_dual_infeasible_low_acc;   /* 1e-12 */
  double eps_primal_infeasible_high_acc, eps_dual_infeasible_high_acc; /* 1e-16 */
  int64_t check_terminate_freq;      /* 2000 */
  int64_t kkt_restart_freq;          /* 2000 */
  int64_t duality_gap_restart_freq;  /* 2000 */
  int32_t use_kkt_restart;           /* 0 */
  int32_t use_duality_gap_restart;   /* 1 */
  int32_t rescaling;     /* 0 none, 1 ruiz, 2 pock_chambolle, 3 ruiz_pock_chambolle (default) */
  int32_t cpu_semantics; /* 0: pdcs_gpu semantics (default); 1: pdcs_cpu acceptance + denominators */
  int32_t threads;       /* OpenMP threads, <=0: all */
  int32_t verbose;
  double time_limit;     /* seconds, <=0 or inf: none */
  int64_t attempt_limit; /* >0: stop after this many PDHG attempts (bounded CPU sample) */
  const double* warm_x;  /* optional warm start (original scale) */
  const double* warm_y;
  int32_t force_resolving; /* test hook: enter the resolving fallback at the first outer iteration */
  int32_t pad;
} oracle_options;

typedef struct {
  double* x;             /* out n (original scale) */
  double* y;             /* out m (original scale) */
  double primal_objective, dual_objective;
  double l_inf_rel_primal_res, l_inf_rel_dual_res, rel_gap;
  double l_2_rel_primal_res, l_2_rel_dual_res;
  int64_t iter, restart_used;
  int32_t exit_code;     /* 0 optimal, 1 max_iter, 2-5 infeasible, 6 time limit, 8 nan, 9 inf, 10 attempt limit */
  int32_t returned_sequence; /* 0 current iterate, 1 averaged iterate */
  double solve_seconds;  /* main loop time (excludes preprocessing, like the reference timer) */
  double setup_seconds;
} oracle_result;

void oracle_default_options(oracle_options* o);
/* Project one block in place.  S: per-element scaling (NULL = ones).
 * lo/hi used by ORC_BOX only.  Returns 0 on success. */
int oracle_project_block(int kind, double* v, int64_t len, const double* S,
                         const double* lo, const double* hi);
/* Euclidean projection onto the exponential cone scaled by D (D o K_exp). */
void oracle_proj_exp_scaled(double* v, const double* D);
int oracle_solve(const oracle_problem* p, const oracle_options* o, oracle_result* r);
/* Shared KKT evaluator of a final point in the original scale (8 outputs, see the .cpp). */
int oracle_evaluate(const oracle_problem* p, const double* x, const double* y, double* out);
/* Apply the Ruiz(10)+Pock-Chambolle(1) preconditioner and return the scaling
 * vectors (Dr: n, Dl: m) and the scaled CSR values (nnz). */
int oracle_precondition(const oracle_problem* p, int rescaling, double* Dr, double* Dl,
                        double* scaled_val);

#ifdef __cplusplus
}
#endif
#endif
