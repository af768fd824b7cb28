// pdcs_tiles.cuh -- instance-tiled SpMV of the batched solver.
//
// The merged matrix is block diagonal: the rows of instance k touch only the
// columns of instance k, at most a few thousand values.  A tile is a range of
// one instance's rows (in the instance's own row order, across its type runs);
// its CTA first stages the instance's whole column segment (x for G, y for G')
// in shared memory, then runs the rows with every gather served from shared
// memory.  Column indices are stored as 16-bit instance-local positions (the
// problem's own column numbers), so a nonzero streams 6 bytes in FP32 and
// 10 in FP64 instead of 8 and 12, and no gather reaches L1 or L2.  Sums run in
// a fixed order: lane-strided partial sums in the matrix's precision, then a
// butterfly in FP64 over the row's lane group.
#pragma once
#include <map>
#include <mutex>

#include "pdcs_batch_kernels.cuh"

namespace pdcs {

constexpr int64_t kTileMaxCols = 65535;  // 16-bit local column indices
// nonzeros a lane loads at once: 16 FP32 values (more bytes in flight per warp),
// 8 FP64 ones (16 doubles per lane spill registers)
template <class T>
constexpr int kTileLN = sizeof(T) == 4 ? 16 : 8;
constexpr int kTileThreads = 512;        // a tile's CTA: 16 warps share one staged column segment
constexpr int kTileWarps = kTileThreads / 32;

struct TileCsr {
  const int32_t* rp;        // merged CSR row pointers
  const uint16_t* cl;       // instance-local column of every nonzero
  const int4* tiles;        // {instance, first row ordinal, end ordinal, lanes per row}
  int64_t ntiles;
  const int32_t* act;       // tiles of the iterating instances (NULL: every tile)
  const int64_t* n_act;
  RunTable rows, cols;      // row-side / column-side runs of every instance
  const int32_t* rloc;      // K * kMaxRuns: instance-local first row of each row run
  const int32_t* cloc;      // K * kMaxRuns: instance-local first column of each column run
  int32_t max_cols;         // the largest instance's column count (staged elements)
};

// Instance-local column of every nonzero: the column's type region gives its run,
// the run's merged start and local start give the local position.
struct RegionStarts {
  int64_t s[kMaxRuns];
};
__global__ void local_cols_kernel(int64_t R, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                  const int32_t* __restrict__ row_inst, RegionStarts reg,
                                  const int64_t* __restrict__ col_run_start, const int32_t* __restrict__ cloc,
                                  uint16_t* __restrict__ out) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < R; i += stride) {
    const int64_t k = row_inst[i];
    for (int32_t e = rp[i]; e < rp[i + 1]; ++e) {
      const int64_t c = ci[e];
      int t = 0;
      for (int q = 1; q < kMaxRuns; ++q)
        if (c >= reg.s[q]) t = q;
      out[e] = (uint16_t)(cloc[k * kMaxRuns + t] + (c - col_run_start[k * kMaxRuns + t]));
    }
  }
}

template <class T, int NV>
using TileVal = std::conditional_t<NV == 1, T, typename Vec2T<T>::type>;

template <class T, int NV>
__device__ __forceinline__ TileVal<T, NV> tile_load(const T* x0, const T* x1, int64_t i) {
  if constexpr (NV == 1) {
    return x0[i];
  } else if constexpr (NV == kPair) {
    return reinterpret_cast<const typename Vec2T<T>::type*>(x0)[i];
  } else {
    typename Vec2T<T>::type v;
    v.x = x0[i];
    v.y = x1[i];
    return v;
  }
}

// y0 = A x0 (and y1 = A x1 for NV 2 / kPair) over the rows of the listed tiles.
// Dynamic shared memory: A.max_cols values of TileVal<T, NV>.
template <class T, int NV>
__global__ void __launch_bounds__(kTileThreads) spmv_tile_kernel(TileCsr A, const T* __restrict__ vals, const T* x0,
                                                             const T* x1, T* y0, T* y1,
                                                             const int32_t* __restrict__ active) {
  if (active && !*active) return;
  using V = TileVal<T, NV>;
  extern __shared__ __align__(16) unsigned char tile_smem[];
  V* sx = reinterpret_cast<V*>(tile_smem);
  __shared__ int64_t run_row[kMaxRuns];
  __shared__ int32_t run_ord[kMaxRuns];
  const int64_t nt = A.act ? *A.n_act : A.ntiles;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t q = blockIdx.x; q < nt; q += gridDim.x) {
    const int4 tl = A.tiles[A.act ? (int64_t)A.act[q] : q];
    const int64_t k = tl.x;
    if (threadIdx.x < kMaxRuns) {
      run_row[threadIdx.x] = A.rows.start[k * kMaxRuns + threadIdx.x];
      run_ord[threadIdx.x] = A.rloc[k * kMaxRuns + threadIdx.x];
    }
    for (int r = 0; r < kMaxRuns; ++r) {
      const int64_t s0 = A.cols.start[k * kMaxRuns + r], L = A.cols.len[k * kMaxRuns + r];
      V* dst = sx + A.cloc[k * kMaxRuns + r];
      for (int64_t i = threadIdx.x; i < L; i += kTileThreads) dst[i] = tile_load<T, NV>(x0, x1, s0 + i);
    }
    __syncthreads();
    const int g = tl.w, gl = lane & (g - 1), per = 32 / g;
    // the loop bound is uniform across the warp (every lane reaches the shuffles)
    for (int64_t ob = tl.y + (int64_t)warp * per; ob < tl.z; ob += (int64_t)kTileWarps * per) {
      const int64_t o = ob + lane / g;
      const bool valid = o < tl.z;
      int64_t row = 0;
      if (valid) {
        int r = 0;
        for (int t = 1; t < kMaxRuns; ++t)  // the last run starting at or before o (empty runs share starts)
          if (o >= run_ord[t]) r = t;
        row = run_row[r] + (o - run_ord[r]);
      }
      const int32_t kb = valid ? A.rp[row] : 0, ke = valid ? A.rp[row + 1] : 0;
      // a lane's partial sums in T (FP32 rows sum in FP32, as the binned kernel's
      // short rows do), widened to FP64 for the lane group's butterfly
      T p0 = T(0), p1 = T(0);
      for (int32_t e0 = kb + gl; e0 < ke; e0 += kTileLN<T> * g) {
        T v[kTileLN<T>];
        uint16_t c[kTileLN<T>];
#pragma unroll
        for (int u = 0; u < kTileLN<T>; ++u) {  // every load of the chunk in flight together
          const int32_t e = e0 + u * g;
          const bool ok = e < ke;
          v[u] = ok ? vals[e] : T(0);
          c[u] = ok ? A.cl[e] : (uint16_t)0;
        }
#pragma unroll
        for (int u = 0; u < kTileLN<T>; ++u) {
          if (e0 + u * g < ke) {
            const V xv = sx[c[u]];
            if constexpr (NV == 1) {
              p0 = fma(v[u], xv, p0);
            } else {
              p0 = fma(v[u], xv.x, p0);
              p1 = fma(v[u], xv.y, p1);
            }
          }
        }
      }
      double a0 = (double)p0, a1 = (double)p1;
      for (int s = g >> 1; s > 0; s >>= 1) {
        a0 += __shfl_xor_sync(kFull, a0, s, g);
        if (NV != 1) a1 += __shfl_xor_sync(kFull, a1, s, g);
      }
      if (valid && gl == 0) {
        y0[row] = (T)a0;
        if (NV != 1) y1[row] = (T)a1;
      }
    }
    __syncthreads();  // the next tile restages sx and the run tables
  }
}

template <class T, int NV>
inline size_t tile_smem_bytes(const TileCsr& A) {
  return sizeof(TileVal<T, NV>) * (size_t)std::max(A.max_cols, 1);
}

// Raise the kernel's dynamic shared memory limit to what A needs.  The
// attribute belongs to the function, not to a solver: it only ever grows, so
// graphs captured by earlier solvers with larger tiles stay launchable.
template <class T, int NV>
inline void tile_prepare(const TileCsr& A) {
  static std::mutex mu;
  static std::map<int, size_t> set;  // per device
  int dev = 0;
  PDCS_CUDA(cudaGetDevice(&dev));
  const size_t need = tile_smem_bytes<T, NV>(A);
  std::lock_guard<std::mutex> lock(mu);
  if (need <= set[dev]) return;
  PDCS_CUDA(cudaFuncSetAttribute(spmv_tile_kernel<T, NV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need));
  set[dev] = need;
}

template <class T, int NV>
inline void launch_spmv_tile(const TileCsr& A, int grid, const T* vals, const std::type_identity_t<T>* x0,
                             const std::type_identity_t<T>* x1, std::type_identity_t<T>* y0,
                             std::type_identity_t<T>* y1, const int32_t* active, cudaStream_t s) {
  spmv_tile_kernel<T, NV><<<grid, kTileThreads, tile_smem_bytes<T, NV>(A), s>>>(A, vals, x0, x1, y0, y1, active);
}

}  // namespace pdcs
