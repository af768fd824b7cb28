/*
 * pdcs_ref_shim.h -- lets g++ compile the reference's scalar CUDA projection
 * code (src/pdcs_gpu/cuda/massive_block_proj.cu, which includes exp_proj.cu)
 * unmodified, as host code, for the test-only library oracle/_ref.
 *
 * TEST INFRASTRUCTURE ONLY: the reference build is a checker for the oracle
 * restatement and for the CUDA projections.  Nothing in the product links it.
 *
 * The kernel massive_block_proj (massive_block_proj.cu:1081-1193) runs every
 * cone block of its table on one thread in a grid-stride loop; with a
 * one-thread "grid" (blockIdx = threadIdx = 0, blockDim = gridDim = 1) the
 * same function is a serial host loop over all blocks.  The CUDA qualifiers
 * are defined away, and min/max/abs get the double overloads CUDA's math
 * headers provide on the device.
 */
#ifndef PDCS_REF_SHIM_H
#define PDCS_REF_SHIM_H
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>

#define __device__
#define __global__
#define __host__
#define __forceinline__ inline

struct pdcs_ref_dim3 {
  unsigned x, y, z;
};
static const pdcs_ref_dim3 threadIdx = {0, 0, 0};
static const pdcs_ref_dim3 blockIdx = {0, 0, 0};
static const pdcs_ref_dim3 blockDim = {1, 1, 1};
static const pdcs_ref_dim3 gridDim = {1, 1, 1};

using std::abs;
using std::exp;
using std::fabs;
using std::fmax;
using std::fmin;
using std::isfinite;
using std::isinf;
using std::isnan;
using std::log;
using std::pow;
using std::sqrt;
static inline double min(double a, double b) { return std::fmin(a, b); }
static inline double max(double a, double b) { return std::fmax(a, b); }

#endif
