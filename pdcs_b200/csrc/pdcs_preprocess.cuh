// pdcs_preprocess.cuh -- one-shot device preprocessing: input checks, the
// transpose G -> G' and the Ruiz (10 passes, l_inf) + Pock-Chambolle
// (alpha = 1) diagonal equilibration of PDCS (src/pdcs_gpu/preprocess.jl:347-591),
// applied as in scale_data! (:300-345):
//   c /= Dr, [bl, bu] *= Dr, G_ij /= (Dl_i Dr_j), h /= Dl.
// Each pass computes the row and column statistics of the current G, then
// scales, exactly as the reference's ruiz_rescaling! / pock_chambolle_rescaling!.
#pragma once
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "pdcs_kernels.cuh"

namespace pdcs {

// error bits of check_inputs_kernel
enum InputError : int32_t { IE_ROWPTR = 1, IE_COLIND = 2, IE_BOUNDS = 4 };

__global__ void check_inputs_kernel(int64_t m, int64_t n, int64_t nnz, int64_t nb, const int32_t* __restrict__ rp,
                                    const int32_t* __restrict__ ci, const double* __restrict__ bl,
                                    const double* __restrict__ bu, int32_t* __restrict__ err) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int32_t e = 0;
  if (tid == 0 && (rp[0] != 0 || (int64_t)rp[m] != nnz)) e |= IE_ROWPTR;
  for (int64_t i = tid; i < m; i += stride)
    if (rp[i + 1] < rp[i]) e |= IE_ROWPTR;
  for (int64_t k = tid; k < nnz; k += stride)
    if (ci[k] < 0 || (int64_t)ci[k] >= n) e |= IE_COLIND;
  for (int64_t j = tid; j < nb; j += stride)
    if (!(bl[j] <= bu[j])) e |= IE_BOUNDS;
  if (e) atomicOr(err, e);
}

// Row index of every nonzero, in two flat passes (a row of any length costs
// the same per nonzero): each nonempty row writes its index at its first
// nonzero (the array zeroed before), then an inclusive max-scan fills the rest.
__global__ void row_start_kernel(int64_t m, const int32_t* __restrict__ rp, int32_t* __restrict__ start) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride)
    if (rp[i] < rp[i + 1]) start[rp[i]] = (int32_t)i;
}

struct MaxI32 {
  __device__ __forceinline__ int32_t operator()(int32_t a, int32_t b) const { return a > b ? a : b; }
};

// nonzero count of every column
__global__ void col_count_kernel(int64_t nnz, const int32_t* __restrict__ ci, int32_t* __restrict__ col_cnt) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += stride) atomicAdd(&col_cnt[ci[k]], 1);
}

__global__ void iota_kernel(int32_t* a, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) a[i] = (int32_t)i;
}

// G' entries from G: colind = row of the source nonzero, value = its value
__global__ void gather_transpose_kernel(int64_t nnz, const int32_t* __restrict__ perm,
                                        const int32_t* __restrict__ row_of, const double* __restrict__ gv,
                                        int32_t* __restrict__ tci, double* __restrict__ tv) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nnz; q += stride) {
    const int32_t k = perm[q];
    tci[q] = row_of[k];
    tv[q] = gv[k];
  }
}

// per row of a CSR (values read through an optional permutation): max |v| or
// sum |v|, a warp per row; rows of more than long_min nonzeros are left to
// row_absstat_long_kernel (long_min < 0: none)
template <bool SUM>
__global__ void row_absstat_kernel(int64_t rows, const int32_t* __restrict__ rp, const double* __restrict__ v,
                                   const int32_t* __restrict__ perm, double* __restrict__ out,
                                   int64_t long_min = -1) {
  const int lane = threadIdx.x & 31;
  const int64_t wstride = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < rows; i += wstride) {
    if (long_min >= 0 && rp[i + 1] - rp[i] > long_min) continue;  // warp-uniform
    double a = 0.0;
    for (int32_t k = rp[i] + lane; k < rp[i + 1]; k += 32) {
      const double x = fabs(perm ? v[perm[k]] : v[k]);
      a = SUM ? a + x : fmax(a, x);
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double b = __shfl_down_sync(kFull, a, o);
      a = SUM ? a + b : fmax(a, b);
    }
    if (lane == 0) out[i] = a;
  }
}

// the same statistic for the long rows listed in `list`, a CTA per row
template <bool SUM>
__global__ void __launch_bounds__(kThreads) row_absstat_long_kernel(int64_t nlist, const int32_t* __restrict__ list,
                                                                    const int32_t* __restrict__ rp,
                                                                    const double* __restrict__ v,
                                                                    const int32_t* __restrict__ perm,
                                                                    double* __restrict__ out) {
  __shared__ double sh[kWarps];
  for (int64_t q = blockIdx.x; q < nlist; q += gridDim.x) {
    const int32_t i = list[q];
    double a = 0.0;
    for (int32_t k = rp[i] + threadIdx.x; k < rp[i + 1]; k += kThreads) {
      const double x = fabs(perm ? v[perm[k]] : v[k]);
      a = SUM ? a + x : fmax(a, x);
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double b = __shfl_down_sync(kFull, a, o);
      a = SUM ? a + b : fmax(a, b);
    }
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = sh[0];
      for (int w = 1; w < kWarps; ++w) t = SUM ? t + sh[w] : fmax(t, sh[w]);
      out[i] = t;
    }
    __syncthreads();
  }
}

// a = 1 where a == 0, sqrt(a) elsewhere
__global__ void sqrt_or_one_kernel(double* a, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    a[i] = (a[i] == 0.0) ? 1.0 : sqrt(a[i]);
}

// G_ij /= (con_i var_j), flat over the nonzeros (row_of: the row of each)
__global__ void scale_matrix_kernel(int64_t nnz, const int32_t* __restrict__ row_of, const int32_t* __restrict__ ci,
                                    double* __restrict__ v, const double* __restrict__ con,
                                    const double* __restrict__ var) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += stride)
    v[k] /= (con[row_of[k]] * var[ci[k]]);
}

// c /= var, Dr *= var, [bl, bu] *= var (box part), h /= con, Dl *= con
__global__ void scale_vectors_kernel(int64_t n, int64_t nb, int64_t m, const double* __restrict__ var,
                                     const double* __restrict__ con, double* __restrict__ c, double* __restrict__ Dr,
                                     double* __restrict__ bl, double* __restrict__ bu, double* __restrict__ h,
                                     double* __restrict__ Dl) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t L = n > m ? n : m;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < L; i += stride) {
    if (i < n) {
      c[i] /= var[i];
      Dr[i] *= var[i];
      if (i < nb) {
        bl[i] *= var[i];
        bu[i] *= var[i];
      }
    }
    if (i < m) {
      h[i] /= con[i];
      Dl[i] *= con[i];
    }
  }
}

// bl_fin / bu_fin (infinities -> 0) and the slack box lambda bounds (gen_lambd,
// src/pdcs_gpu/def_rpdhg_gen.jl:5-17)
__global__ void box_aux_kernel(int64_t nb, const double* __restrict__ bl, const double* __restrict__ bu,
                               double* __restrict__ bl_fin, double* __restrict__ bu_fin,
                               double* __restrict__ lam_l, double* __restrict__ lam_u) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const double inf = __longlong_as_double(0x7ff0000000000000LL);
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nb; j += stride) {
    const double l = bl[j], u = bu[j];
    bl_fin[j] = isinf(l) ? 0.0 : l;
    bu_fin[j] = isinf(u) ? 0.0 : u;
    lam_l[j] = (u == inf) ? 0.0 : -inf;
    lam_u[j] = (l == -inf) ? 0.0 : inf;
  }
}

__global__ void fill_kernel(double* a, double v, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) a[i] = v;
}

// dst[q] = src[idx[q]]
__global__ void gather_kernel(double* __restrict__ dst, const double* __restrict__ src,
                              const int32_t* __restrict__ idx, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) dst[q] = src[idx[q]];
}

__global__ void mul_kernel(double* a, const double* b, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) a[i] *= b[i];
}

}  // namespace pdcs
