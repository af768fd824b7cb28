/*
 * ref_proj.cpp -- host build of the reference's own cone projections
 * (TEST INFRASTRUCTURE ONLY; output oracle/_ref/libpdcs_ref_proj.so).
 *
 * Compiles src/pdcs_gpu/cuda/massive_block_proj.cu of the reference, which
 * includes src/pdcs_gpu/cuda/exp_proj.cu, from where it lies, unmodified,
 * through pdcs_ref_shim.h.  The reference's thread-per-cone kernel
 * massive_block_proj (massive_block_proj.cu:1081-1193) then runs as a serial
 * loop over the blocks, dispatching on the same projection codes (0-29) to
 *   soc_proj            :221   (codes 5, 7, 20, 21)
 *   soc_proj_diagonal   :606   (6, 22)
 *   rsoc_proj           :318   (8, 10, 23, 24)
 *   rsoc_proj_diagonal  :871   (9, 25)
 *   exponent_proj(_diagonal), dualExponent_proj(_diagonal)
 *                       exp_proj.cu:706, :757, :966, :955   (11-16, 26-29)
 * and the box / zero / nonnegative loops of blocks 0 and 1.
 *
 * The arrays are the ones the Julia host passes (def_rpdhg_gen.jl:59, :411):
 * D_scaled = Dr_product_inv_normalized (S0/S_i for SOC, sqrt(S0 S1)/S_i for
 * RSOC, 1/S_i for the exponential cones), D_scaled_squared its square, and
 * two scratch vectors of the array's length; t_warm_start one value per block.
 */
#include "pdcs_ref_shim.h"
#include "massive_block_proj.cu"

extern "C" int pdcs_ref_block_proj(double* arr, double* bl, double* bu, double* D_scaled,
                                   double* D_scaled_squared, double* scratch1, double* scratch2,
                                   double* t_warm_start, const long* head_start, const long* ns,
                                   int blkNum, long* proj_type, double abs_tol, double rel_tol) {
  massive_block_proj(arr, bl, bu, D_scaled, D_scaled_squared, scratch1, scratch2, t_warm_start,
                     head_start, ns, blkNum, proj_type, abs_tol, rel_tol);
  return 0;
}
