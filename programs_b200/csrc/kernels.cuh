// kernels.cuh -- sm_100a kernels of the face-addressed Krylov solvers.
//
// Storage (built on the host by solv_gpu.cu):
//   * cells live in an internal order: wavefront level of the lower-
//     triangular DAG first, then the caller's index, so every level of the
//     DIC/DILU sweeps is one contiguous range and "neighbour j is below
//     cell i in the caller's order" is exactly "j < i" internally;
//   * each cell's interior faces form one row of a sliced ELL (32 cells per
//     slice, slot-major inside a slice, so a warp reads 32 consecutive
//     words per slot); slots keep the cell's faces in ascending face order,
//     which is the order the reference's face loop adds them in;
//   * vectors with V components are cell-interleaved: x[i*V + v].
// FP64 arithmetic uses explicit _rn intrinsics (no FMA contraction), so
// matrix products, residuals and sweeps are bit-identical to the in-order
// CPU restatement; reductions use a fixed tree and are run-to-run
// deterministic.
#pragma once
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace sg {

constexpr double kSmall = 1e-20;  // spray-simulation/precision.f90:8
constexpr double kLarge = 1e20;   // spray-simulation/precision.f90:9
constexpr int kWarp = 32;

// ---- precision helpers ---------------------------------------------------
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return a * b; }
__device__ __forceinline__ float add(float a, float b) { return a + b; }
__device__ __forceinline__ float sub(float a, float b) { return a - b; }
// Reduction term: always formed and accumulated in FP64.
__device__ __forceinline__ double prod(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double prod(float a, float b) { return __dmul_rn((double)a, (double)b); }

// ---- per (system, component) Krylov state ---------------------------------
struct Lane {
  double s, beta, alpha, pq;           // CG: s = r.z, beta, alpha
  double rho, beta0, gam, omeg;        // BiCGSTAB (alpha shared)
  double res0_n, ratio, reduc, l1;
  double gs;                           // FCG: residual scale fed to the network
  double s_prev;                       // CG: r.z of the previous iteration
  double l1_stop;                      // FP32 inner iterations: stop for a reliable
                                       // update once |r|_1 falls below this (0: never)
  int iter, n_iter, active, status;
};
enum : int { kLaneRunning = 0, kLaneConverged = 1, kLaneMaxIter = 2, kLaneNaN = 3,
             kLaneStall = 4, kLaneRefine = 5 };

// Flexible-CG beta = -(z.q)/(p.q) for the next direction p = z + beta p,
// restarted (beta = 0) each time the lane has taken a multiple of n
// iterations on its n-cell system.  CG ends within n steps in exact
// arithmetic; past them the old direction only cancels the new one (on a
// one-cell system z + beta p is exactly zero and the iteration stops
// moving).  Systems with more cells than iterations never restart.
__device__ __forceinline__ double flex_beta(const Lane& L, double zq, int n) {
  return (L.pq > 0.0 && L.iter % n != 0) ? -zq / L.pq : 0.0;
}

// The step scalars of the FP32 inner iterations (mixed precision) divide
// without the reference's absolute guard `+ small` (precision.f90:8): after
// a reliable update the residual of a small or weakly driven system, and
// with it every inner product, can lie far below 1e-20, where the guard
// would shrink each step towards zero and the iteration would stall.  A
// zero denominator gives a zero step.  The FP64 kernels keep the
// reference's expressions unchanged.
__device__ __forceinline__ double div0(double num, double den) {
  return den != 0.0 ? num / den : 0.0;
}

template <typename T>
struct Rows {
  const int* __restrict__ slice_ptr;    // element offset of each slice
  const uint8_t* __restrict__ slice_w;  // slots in each slice
  const int* __restrict__ col;          // internal column, -1 = padding
  const T* __restrict__ val;            // A(i, col) for the matrix product
  const T* __restrict__ sval;           // sweep coefficient (ng%n below, ng%p above)
  const T* __restrict__ diag;           // pl
};

// Reduction geometry: each block works on one segment (system) and strides
// through that segment's cells; partial sums go to part[], and the last
// block of a segment to finish (ticket) combines them in block order.
struct SegMap {
  const int* __restrict__ blk_seg;
  const int* __restrict__ blk_rank;
  const int* __restrict__ seg_nblk;
  const int* __restrict__ seg_blk0;
  const int* __restrict__ seg_c0;
  const int* __restrict__ seg_c1;
  unsigned int* ticket;
  int* n_active;  // lanes still iterating (host polls this)
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of NR values; result valid in thread 0.  Fixed order.
template <int NR>
__device__ __forceinline__ void block_sum(double (&v)[NR]) {
  __shared__ double sh[NR][32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < NR; ++k) v[k] = warp_sum(v[k]);
  if (l == 0) {
#pragma unroll
    for (int k = 0; k < NR; ++k) sh[k][w] = v[k];
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      double t = l < nw ? sh[k][l] : 0.0;
      v[k] = warp_sum(t);
    }
  }
  __syncthreads();
}

// Commit this block's partials; returns true in the segment's last block,
// with the segment totals in tot[] (valid in every thread of that block).
template <int NR>
__device__ __forceinline__ bool seg_commit(const SegMap& sm, int b, int s,
                                           double* __restrict__ part,
                                           double (&v)[NR], double (&tot)[NR]) {
  __shared__ bool last;
  __shared__ double tsh[NR];
  block_sum<NR>(v);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NR; ++k) part[(size_t)b * NR + k] = v[k];
    __threadfence();
    unsigned t = atomicAdd(&sm.ticket[s], 1u);
    last = (t == (unsigned)sm.seg_nblk[s] - 1u);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  const int nb = sm.seg_nblk[s], b0 = sm.seg_blk0[s];
  double acc[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) acc[k] = 0.0;
  for (int j = threadIdx.x; j < nb; j += blockDim.x) {
#pragma unroll
    for (int k = 0; k < NR; ++k) acc[k] += __ldcg(&part[(size_t)(b0 + j) * NR + k]);
  }
  block_sum<NR>(acc);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NR; ++k) tsh[k] = acc[k];
    sm.ticket[s] = 0u;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NR; ++k) tot[k] = tsh[k];
  return true;
}

__device__ __forceinline__ void lane_stop(Lane& L, int status, int* n_active) {
  if (L.active) {
    L.active = 0;
    L.status = status;
    atomicSub(n_active, 1);
  }
}

// Kernels on the reduction grid (SegMap) are meant to run every block of the
// grid at once: the grid holds at most 2048 threads per SM (blocks of at
// most 256 threads), and the register budget of the one-component kernels
// is capped at 32 so that all of them are resident -- a block left for a
// second wave would run the tail of every reduction at a fraction of the
// occupancy.  Several components (V > 1) get 64 registers and run in two
// full waves.
constexpr int kMaxBlock = 256;
#define SG_BOUNDS(V) __launch_bounds__(sg::kMaxBlock, ((V) == 1 ? 8 : 4))

// Row walk helpers ---------------------------------------------------------
template <typename T>
struct RowIt {
  int base, w;
  __device__ __forceinline__ RowIt(const Rows<T>& R, int i) {
    const int sl = i >> 5;
    base = __ldg(&R.slice_ptr[sl]) + (i & 31);
    w = __ldg(&R.slice_w[sl]);
  }
};

// y = A x for V interleaved components.
// FP64: y_i = pl_i x_i + sum in face order (the reference's arithmetic).
// FP32: difference form y_i = rs_i x_i + sum_j a_ij (x_j - x_i), where the
// FP32 "diagonal" holds the row sum rs_i = pl_i + sum_j a_ij (formed in
// FP64).  For the smooth vectors late Krylov iterations produce, x_j - x_i
// is exact and small, so the product keeps its relative accuracy instead of
// losing log10(cond) digits to cancellation; same bytes moved.
// Rows are walked a chunk of slots at a time: the column indices, the
// coefficients and the gathered x of a chunk are all loaded before any of
// them is used, so a warp keeps several independent gathers in flight; the
// sums still run slot by slot in face order, so the FP64 product stays bit
// for bit the reference's.  FP32 takes 4 slots at a time (0.52 -> 0.69 of
// copy bandwidth); FP64 one: two slots spilled under the reduction
// kernels' 32-register cap and made the FP64 products slower at 256^3
// (0.30 -> 0.38 ms for y = A x, 0.289 -> 0.306 ms for the CG product).
#ifndef SG_ROW_CHUNK64
#define SG_ROW_CHUNK64 1
#endif
constexpr int kRowChunk = 4;
constexpr int kRowChunk64 = SG_ROW_CHUNK64;

template <typename T, int V, int CH = kRowChunk>
__device__ __forceinline__ void row_apply(const Rows<T>& R, int i,
                                          const T* __restrict__ x, T (&y)[V]) {
  RowIt<T> it(R, i);
  const T d = R.diag[i];
  if constexpr (sizeof(T) == 4) {
    T xi[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      xi[v] = x[(size_t)i * V + v];
      y[v] = d * xi[v];
    }
    for (int k0 = 0; k0 < it.w; k0 += CH) {
      int j[CH];
      T a[CH], xv[CH][V];
#pragma unroll
      for (int u = 0; u < CH; ++u) {
        j[u] = -1;
        a[u] = T(0);
        if (k0 + u < it.w) {
          const int e = it.base + (k0 + u) * kWarp;
          j[u] = __ldg(&R.col[e]);
          a[u] = R.val[e];
        }
      }
#pragma unroll
      for (int u = 0; u < CH; ++u)
#pragma unroll
        for (int v = 0; v < V; ++v) xv[u][v] = j[u] >= 0 ? x[(size_t)j[u] * V + v] : xi[v];
#pragma unroll
      for (int u = 0; u < CH; ++u)
        if (j[u] >= 0) {
#pragma unroll
          for (int v = 0; v < V; ++v) y[v] = fmaf(a[u], xv[u][v] - xi[v], y[v]);
        }
    }
  } else {
#pragma unroll
    for (int v = 0; v < V; ++v) y[v] = mul(d, x[(size_t)i * V + v]);
    constexpr int C = V == 1 ? kRowChunk64 : 1;
    for (int k0 = 0; k0 < it.w; k0 += C) {
      int j[C];
      T a[C], xv[C][V];
#pragma unroll
      for (int u = 0; u < C; ++u) {
        j[u] = -1;
        a[u] = T(0);
        if (k0 + u < it.w) {
          const int e = it.base + (k0 + u) * kWarp;
          j[u] = __ldg(&R.col[e]);
          a[u] = R.val[e];
        }
      }
#pragma unroll
      for (int u = 0; u < C; ++u)
#pragma unroll
        for (int v = 0; v < V; ++v) xv[u][v] = j[u] >= 0 ? x[(size_t)j[u] * V + v] : T(0);
#pragma unroll
      for (int u = 0; u < C; ++u)
        if (j[u] >= 0) {
#pragma unroll
          for (int v = 0; v < V; ++v) y[v] = add(y[v], mul(a[u], xv[u][v]));
        }
    }
  }
}

// FP32 row-sum "diagonal" for the difference-form product: rs_i = pl_i +
// sum_j a_ij, formed in FP64 then rounded once.
__global__ void k_rowsum_diag(int n, Rows<double> R, float* __restrict__ rs) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    RowIt<double> it(R, i);
    double s = R.diag[i];
    for (int k = 0; k < it.w; ++k) {
      const int e = it.base + k * kWarp;
      if (R.col[e] >= 0) s += R.val[e];
    }
    rs[i] = (float)s;
  }
}

// ---- layout conversion ---------------------------------------------------
// caller phi (cell-major [N][V], caller order) -> internal interleaved
template <typename T>
__global__ void k_phi_in(int n, int V, const int* __restrict__ old_of_new,
                         const double* __restrict__ src, T* __restrict__ dst) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int o = old_of_new[i];
    for (int v = 0; v < V; ++v) dst[(size_t)i * V + v] = (T)src[(size_t)o * V + v];
  }
}
template <typename T>
__global__ void k_phi_out(int n, int V, const int* __restrict__ old_of_new,
                          const T* __restrict__ src, double* __restrict__ dst) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int o = old_of_new[i];
    for (int v = 0; v < V; ++v) dst[(size_t)o * V + v] = (double)src[(size_t)i * V + v];
  }
}
// caller res0 (column-major [V][N]) <-> internal interleaved
__global__ void k_col_in(int n, int V, const int* __restrict__ old_of_new,
                         const double* __restrict__ src, double* __restrict__ dst) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int o = old_of_new[i];
    for (int v = 0; v < V; ++v) dst[(size_t)i * V + v] = src[(size_t)v * n + o];
  }
}
__global__ void k_col_out(int n, int V, const int* __restrict__ old_of_new,
                          const double* __restrict__ src, double* __restrict__ dst) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int o = old_of_new[i];
    for (int v = 0; v < V; ++v) dst[(size_t)v * n + o] = src[(size_t)i * V + v];
  }
}

// ---- matrix values ---------------------------------------------------------
// slot_src = 2*face + (1 if the row's cell is the face neighbour), -1 pad.
// val: the coefficient the face loop multiplies x(other cell) by for this
// row (ng%p for the owner's row, ng%n for the neighbour's row);
// sval: the sweep coefficient, ng%n for a lower neighbour, ng%p for an
// upper one (solv_direct.f90:19,33).
template <typename T>
__global__ void k_fill_values(int n, const int* __restrict__ slice_ptr,
                              const uint8_t* __restrict__ slice_w,
                              const int* __restrict__ slot_src, const int* __restrict__ col,
                              const double* __restrict__ p, const double* __restrict__ nn,
                              T* __restrict__ val, T* __restrict__ sval) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int sl = i >> 5, base = slice_ptr[sl] + (i & 31), w = slice_w[sl];
    for (int k = 0; k < w; ++k) {
      const int e = base + k * kWarp;
      const int s = slot_src[e];
      if (s < 0) {
        val[e] = (T)0;
        if (sval) sval[e] = (T)0;
        continue;
      }
      const int f = s >> 1;
      val[e] = (T)((s & 1) ? nn[f] : p[f]);
      if (sval) sval[e] = (T)(col[e] < i ? nn[f] : p[f]);
    }
  }
}
template <typename T>
__global__ void k_fill_diag(int n, const int* __restrict__ old_of_new,
                            const double* __restrict__ pl, T* __restrict__ diag) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    diag[i] = (T)pl[old_of_new[i]];
}
template <typename Tsrc, typename Tdst>
__global__ void k_convert(long long n, const Tsrc* __restrict__ a, Tdst* __restrict__ b) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x)
    b[e] = (Tdst)a[e];
}

// ---- residual: solv_res.f90:12-29 ----------------------------------------
// r_i = ((b_i - pl_i phi_i) - a_1 phi_j1) - ...; L1 norm per component.
template <int V>
__global__ void SG_BOUNDS(V) k_res(Rows<double> R, SegMap sm, const double* __restrict__ phi,
                      double* __restrict__ r, int not_r0, double* __restrict__ part,
                      double* __restrict__ l1_out) {
  const int b = blockIdx.x, s = sm.blk_seg[b];
  const int c0 = sm.seg_c0[s], c1 = sm.seg_c1[s];
  const int stride = sm.seg_nblk[s] * blockDim.x;
  double l1[V];
#pragma unroll
  for (int v = 0; v < V; ++v) l1[v] = 0.0;
  for (int i = c0 + sm.blk_rank[b] * blockDim.x + threadIdx.x; i < c1; i += stride) {
    double y[V];
    if (!not_r0) {
      RowIt<double> it(R, i);
      const double d = R.diag[i];
#pragma unroll
      for (int v = 0; v < V; ++v) y[v] = sub(r[(size_t)i * V + v], mul(d, phi[(size_t)i * V + v]));
      for (int k = 0; k < it.w; ++k) {
        const int e = it.base + k * kWarp;
        const int j = __ldg(&R.col[e]);
        if (j >= 0) {
          const double a = R.val[e];
#pragma unroll
          for (int v = 0; v < V; ++v) y[v] = sub(y[v], mul(a, phi[(size_t)j * V + v]));
        }
      }
#pragma unroll
      for (int v = 0; v < V; ++v) r[(size_t)i * V + v] = y[v];
    } else {
#pragma unroll
      for (int v = 0; v < V; ++v) y[v] = r[(size_t)i * V + v];
    }
#pragma unroll
    for (int v = 0; v < V; ++v) l1[v] += fabs(y[v]);
  }
  double tot[V];
  if (seg_commit<V>(sm, b, s, part, l1, tot) && threadIdx.x == 0) {
#pragma unroll
    for (int v = 0; v < V; ++v) l1_out[s * V + v] = tot[v];
  }
}

__global__ void k_set_res0n(Lane* lanes, int nl, const double* __restrict__ l1) {
  for (int l = threadIdx.x; l < nl; l += blockDim.x) lanes[l].res0_n = l1[l];
}

// ---- mixed precision: FP32 inner solve inside FP64 refinement --------------
// inner right-hand side r_f = (float) r, shadow r0_f = r_f, correction d = 0
template <int V>
__global__ void k_mp_start(long long nv, const double* __restrict__ r, float* __restrict__ rf,
                           float* __restrict__ r0f, float* __restrict__ d) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nv;
       e += (long long)gridDim.x * blockDim.x) {
    const float t = (float)r[e];
    rf[e] = t;
    r0f[e] = t;
    d[e] = 0.0f;
  }
}
__global__ void k_add(long long n, double* __restrict__ x, const double* __restrict__ y) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x)
    x[e] += y[e];
}
// phi += (double) d for the (system, component) lanes flagged in mask
// (FP64 solution accumulation)
template <int V>
__global__ void SG_BOUNDS(V) k_mp_accum(SegMap sm, const int* __restrict__ mask, double* __restrict__ phi,
                           const float* __restrict__ d) {
  const int b = blockIdx.x, s = sm.blk_seg[b];
  bool on[V];
  bool any = false;
#pragma unroll
  for (int v = 0; v < V; ++v) { on[v] = mask[s * V + v] != 0; any |= on[v]; }
  if (!any) return;
  const int c0 = sm.seg_c0[s], c1 = sm.seg_c1[s];
  const int stride = sm.seg_nblk[s] * blockDim.x;
  for (int i = c0 + sm.blk_rank[b] * blockDim.x + threadIdx.x; i < c1; i += stride) {
#pragma unroll
    for (int v = 0; v < V; ++v)
      if (on[v]) phi[(size_t)i * V + v] += (double)d[(size_t)i * V + v];
  }
}

// ---- sync-free triangular recurrences ---------------------------------------
// solv_precond (the DIC/DILU factorisation) and solv_direct (the two
// triangular sweeps) are recurrences over the cells: in the internal order
// every lower neighbour of a cell has a lower index (and every upper one a
// higher index), so a cell can be computed as soon as the values of its
// lower (forward) or upper (backward) neighbours exist.  One cooperative
// launch does a whole recurrence: warp w of W owns the 32-cell slices
// w, w + W, w + 2W, ... (backward: counted from the top) and takes them in
// that order; the output array starts out filled with a signalling-NaN
// pattern ("pending"), which arithmetic never produces (it returns quiet
// NaNs), and a cell reads a neighbour's value with a relaxed load until it
// is no longer pending.  All warps are resident at once (cooperative
// launch), so the lowest unfinished slice always has its owner running and
// its inputs done: the recurrence cannot deadlock.  Each cell still adds its
// neighbour terms one by one in slot (face) order, with the reference's
// operations, so the results are bit for bit those of the sequential loops.
// Every wait is bounded (kSweepPolls polls): a wait that runs out sets
// SweepCtl::err, every warp then stops waiting, and the host reports the
// error and refills the pending state before the next sweep.
struct SweepCtl {
  int err;      // a wait ran out (sticky until the host clears it)
  int pad[3];
};
constexpr int kSweepPolls = 1 << 20;
constexpr int kSweepThreads = 256;

template <typename T> struct Pending;
template <> struct Pending<double> {
  using U = unsigned long long;
  static constexpr U bits = 0x7ff5a5a5a5a5a5a5ull;  // signalling NaN
  static __device__ __forceinline__ double value() { return __longlong_as_double((long long)bits); }
  static __device__ __forceinline__ double from(U u) { return __longlong_as_double((long long)u); }
};
template <> struct Pending<float> {
  using U = unsigned int;
  static constexpr U bits = 0x7fa5a5a5u;  // signalling NaN
  static __device__ __forceinline__ float value() { return __int_as_float((int)bits); }
  static __device__ __forceinline__ float from(U u) { return __int_as_float((int)u); }
};

__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned int ld_relaxed(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed(double* p, double v) {
  asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(__double_as_longlong(v))
               : "memory");
}
__device__ __forceinline__ void st_relaxed(float* p, float v) {
  asm volatile("st.relaxed.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(__float_as_int(v)) : "memory");
}
__device__ __forceinline__ int ld_err(const SweepCtl* ctl) {
  return (int)ld_relaxed(reinterpret_cast<const unsigned int*>(&ctl->err));
}

// v = *p once it is no longer pending
template <typename T>
__device__ __forceinline__ bool take(const T* p, T& v) {
  using P = Pending<T>;
  const typename P::U u = ld_relaxed(reinterpret_cast<const typename P::U*>(p));
  v = P::from(u);
  return u != P::bits;
}

// x[0 .. n) = pending
template <typename T>
__global__ void k_fill_pending(long long n, T* __restrict__ x) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x)
    x[e] = Pending<T>::value();
}

// Warp-level driver of one recurrence.  `step(i, k, first)` advances cell i
// (this lane's) from slot k as far as its inputs allow and returns the next
// slot (w when the cell is done and stored).  Slices are taken in the order
// that makes every dependency point to an earlier (or the same) slice.  A
// warp whose lanes wait spins for kSweepSpin polls, then sleeps briefly
// between polls.
constexpr int kSweepSpin = 64;
constexpr int kSweepSleep = 64;  // ns

template <bool UP, typename Step>
__device__ __forceinline__ void sweep_slices(int n, const uint8_t* __restrict__ slice_w,
                                             SweepCtl* ctl, Step&& step) {
  const int lane = threadIdx.x & 31;
  const int ns = (n + 31) >> 5;
  const int W = gridDim.x * (blockDim.x >> 5);
  const int gw = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  for (int r = gw; r < ns; r += W) {
    const int s = UP ? ns - 1 - r : r;
    const int i = s * 32 + lane;
    const int w = __ldg(&slice_w[s]);
    int k = step(i, i < n ? 0 : w, true);
    for (int poll = 0;; ++poll) {
      __syncwarp();
      if (__all_sync(0xffffffffu, k >= w)) break;
      if (poll >= kSweepPolls || ((poll & 63) == 63 && ld_err(ctl))) {
        if (lane == 0) atomicExch(&ctl->err, 1);
        break;
      }
      if (poll >= kSweepSpin) __nanosleep(kSweepSleep);
      if (k < w) k = step(i, k, false);
    }
  }
}

// One advance of a recurrence row: from slot k, the slots of the dependency
// side (`dep(j)`) are taken in chunks of C -- their neighbour values and
// their coefficients (`coef(e)`, read-only data) loaded at once, so that a
// coefficient never waits behind a value that has just arrived -- then
// added in slot order up to the first one still pending.  `use(a, xv)`
// folds a ready value in.  Returns the slot to resume from (w when the row
// is complete).
template <int C, int V, typename T, typename Dep, typename Coef, typename Use>
__device__ __forceinline__ int advance(const Rows<T>& R, int base, int w, int k, const T* vals,
                                       Dep&& dep, Coef&& coef, Use&& use) {
  using A = decltype(coef(0));
  while (k < w) {
    int j[C];
    A a[C];
    T xv[C][V];
    bool rdy[C];
#pragma unroll
    for (int u = 0; u < C; ++u) {
      const int e = base + (k + u) * kWarp;
      j[u] = k + u < w ? __ldg(&R.col[e]) : -1;
      rdy[u] = true;
      if (j[u] >= 0 && dep(j[u])) {
        a[u] = coef(e);
#pragma unroll
        for (int v = 0; v < V; ++v) rdy[u] &= take(&vals[(size_t)j[u] * V + v], xv[u][v]);
      }
    }
#pragma unroll
    for (int u = 0; u < C; ++u) {
      if (k >= w) return w;
      if (j[u] >= 0 && dep(j[u])) {
        if (!rdy[u]) return k;
        use(a[u], xv[u]);
      }
      ++k;
    }
  }
  return k;
}

// solv_precond.f90:10-29: d_i = pl_i - sum_{j<i} n^2 c_j (DIC, imat 1) or
// - (p c_j) n (DILU, imat 2) in face order; c_r = d; c = 1/(d + small).
// imat <= 0 is Jacobi (no recurrence; k_precond_jacobi), imat >= 3 keeps
// d = pl (the reference's fall-through).  c must start out pending.
__global__ void __launch_bounds__(kSweepThreads) k_precond_sf(
    int n, int imat, Rows<double> R, const int* __restrict__ slot_src,
    const double* __restrict__ fp, const double* __restrict__ fn, double* c,
    double* __restrict__ c_r, SweepCtl* ctl) {
  const int lane = threadIdx.x & 31;
  double d = 0.0;
  int base = 0;
  sweep_slices<false>(n, R.slice_w, ctl, [&](int i, int k, bool first) -> int {
    const int w = __ldg(&R.slice_w[i >> 5]);
    if (first) {
      if (i >= n) return w;
      base = __ldg(&R.slice_ptr[i >> 5]) + lane;
      d = R.diag[i];
    }
    if (imat == 1 || imat == 2) {
      k = advance<4, 1>(
          R, base, w, k, c, [&](int j) { return j < i; },
          [&](int e) {
            const int f = __ldg(&slot_src[e]) >> 1;
            return make_double2(__ldg(imat == 1 ? &fn[f] : &fp[f]), __ldg(&fn[f]));
          },
          [&](const double2& a, const double (&cj)[1]) {
            if (imat == 1)
              d = sub(d, mul(mul(a.y, a.y), cj[0]));
            else
              d = sub(d, mul(mul(a.x, cj[0]), a.y));
          });
      if (k < w) return k;
    }
    c_r[i] = d;
    st_relaxed(&c[i], 1.0 / add(d, kSmall));
    return w;
  });
}

// Jacobi diagonal (solv_precond.f90:13 with imat <= 0): c_r = pl, c = 1/(pl+small)
__global__ void k_precond_jacobi(int n, const double* __restrict__ diag, double* __restrict__ c,
                                 double* __restrict__ c_r) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double d = diag[i];
    c_r[i] = d;
    c[i] = 1.0 / add(d, kSmall);
  }
}

// slots per chunk: fewer for wide FP64 rows, which would spill
template <typename T, int V> struct SweepChunk {
  static constexpr int value = V == 1 ? 4 : (V >= 4 && sizeof(T) == 8 ? 1 : 2);
};

// solv_direct.f90:12-24 forward sweep, x_i = (b_i - sum_{j<i} n x_j) c_i, into
// t (which starts out pending); the backward sweep's output x is reset to
// pending on the way.
template <typename T, int V>
__global__ void __launch_bounds__(kSweepThreads, 4) k_fwd_sf(
    int n, Rows<T> R, const T* __restrict__ c, const T* __restrict__ bvec, T* t, T* x,
    SweepCtl* ctl, const int* __restrict__ n_active) {
  if (n_active && *n_active == 0) return;
  const int lane = threadIdx.x & 31;
  T acc[V], ci = T(0);
  int base = 0;
  sweep_slices<false>(n, R.slice_w, ctl, [&](int i, int k, bool first) -> int {
    const int w = __ldg(&R.slice_w[i >> 5]);
    if (first) {
      if (i >= n) return w;
      base = __ldg(&R.slice_ptr[i >> 5]) + lane;
      ci = __ldg(&c[i]);
#pragma unroll
      for (int v = 0; v < V; ++v) acc[v] = bvec[(size_t)i * V + v];
    }
    k = advance<SweepChunk<T, V>::value, V>(
        R, base, w, k, t, [&](int j) { return j < i; },
        [&](int e) { return __ldg(&R.sval[e]); },
        [&](const T a, const T (&xv)[V]) {
#pragma unroll
          for (int v = 0; v < V; ++v) acc[v] = sub(acc[v], mul(a, xv[v]));
        });
    if (k < w) return k;
#pragma unroll
    for (int v = 0; v < V; ++v) {
      st_relaxed(&t[(size_t)i * V + v], mul(acc[v], ci));
      x[(size_t)i * V + v] = Pending<T>::value();
    }
    return w;
  });
}

// solv_direct.f90:26-38 backward sweep with the x = x c_r scaling of :26:
// x_i = (t_i c_r_i - sum_{j>i} p x_j) c_i; x starts out pending, and each
// t_i is reset to pending once read, ready for the next forward sweep.
template <typename T, int V>
__global__ void __launch_bounds__(kSweepThreads, 4) k_bwd_sf(
    int n, Rows<T> R, const T* __restrict__ c, const T* __restrict__ c_r, T* t, T* x,
    SweepCtl* ctl, const int* __restrict__ n_active) {
  if (n_active && *n_active == 0) return;
  const int lane = threadIdx.x & 31;
  T acc[V], ci = T(0);
  int base = 0;
  sweep_slices<true>(n, R.slice_w, ctl, [&](int i, int k, bool first) -> int {
    const int w = __ldg(&R.slice_w[i >> 5]);
    if (first) {
      if (i >= n) return w;
      base = __ldg(&R.slice_ptr[i >> 5]) + lane;
      ci = __ldg(&c[i]);
      const T cr = c_r[i];
#pragma unroll
      for (int v = 0; v < V; ++v) acc[v] = mul(t[(size_t)i * V + v], cr);
    }
    k = advance<SweepChunk<T, V>::value, V>(
        R, base, w, k, x, [&](int j) { return j > i; },
        [&](int e) { return __ldg(&R.sval[e]); },
        [&](const T a, const T (&xv)[V]) {
#pragma unroll
          for (int v = 0; v < V; ++v) acc[v] = sub(acc[v], mul(a, xv[v]));
        });
    if (k < w) return k;
#pragma unroll
    for (int v = 0; v < V; ++v) {
      st_relaxed(&x[(size_t)i * V + v], mul(acc[v], ci));
      t[(size_t)i * V + v] = Pending<T>::value();
    }
    return w;
  });
}

// Jacobi: x = b*c (solv_direct.f90:41)
template <typename T, int V>
__global__ void k_jacobi(int n, const T* __restrict__ c, const T* __restrict__ bvec,
                         T* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const T ci = c[i];
#pragma unroll
    for (int v = 0; v < V; ++v) x[(size_t)i * V + v] = mul(bvec[(size_t)i * V + v], ci);
  }
}

// ---- plain matrix product (benchmarks / solv_gpu_spmv) ---------------------
template <typename T, int V>
__global__ void k_spmv(int n, Rows<T> R, const T* __restrict__ x, T* __restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    T t[V];
    row_apply<T, V>(R, i, x, t);
#pragma unroll
    for (int v = 0; v < V; ++v) y[(size_t)i * V + v] = t[v];
  }
}

// ======================= CG: solv_cg.f90:26-84 =============================
// Lane init for CG: s = large, iter = 0, active = 1.
__global__ void k_lane_init(Lane* lanes, int nl, int n_iter, double reduc, int* n_active) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= nl) return;
  Lane L;
  L.s = kLarge; L.beta = 0.0; L.alpha = 1.0; L.pq = 0.0;   // solv_cg.f90:29
  L.rho = 0.0; L.beta0 = 1.0; L.gam = 1.0; L.omeg = 0.0;   // solv_bicg.f90:31-33
  L.res0_n = lanes[l].res0_n;
  L.ratio = 0.0; L.reduc = reduc; L.l1 = 0.0;
  L.iter = 0; L.n_iter = n_iter; L.active = 1; L.status = kLaneRunning; L.l1_stop = 0.0;
  if (n_iter <= 0) { L.active = 0; L.status = kLaneMaxIter; }  // n_active set by the host
  lanes[l] = L;
}

// s = r.z with z = M^-1 r (Jacobi: z = c r, computed here); then
// beta = (1/s_old) s, s_old = s  (solv_cg.f90:44-50).
// FLEX (the FP32 inner iteration, not the reference's): beta = -(z.q)/(p.q)
// with q = A p of the previous step, the flexible-CG formula that
// A-orthogonalises the new direction against the last one explicitly.
template <typename T, int V, bool JAC, bool FLEX = false>
__global__ void SG_BOUNDS(V) k_cg_rz(SegMap sm, const T* __restrict__ c, const T* __restrict__ r,
                        const T* __restrict__ z, double* __restrict__ part,
                        Lane* __restrict__ lanes, const T* __restrict__ q = nullptr) {
  const int b = blockIdx.x, s = sm.blk_seg[b];
  bool any = false;
#pragma unroll
  for (int v = 0; v < V; ++v) any |= lanes[s * V + v].active != 0;
  if (!any) return;
  const int c0 = sm.seg_c0[s], c1 = sm.seg_c1[s];
  const int stride = sm.seg_nblk[s] * blockDim.x;
  double acc[V];
#pragma unroll
  for (int v = 0; v < V; ++v) acc[v] = 0.0;
  for (int i = c0 + sm.blk_rank[b] * blockDim.x + threadIdx.x; i < c1; i += stride) {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const T ri = r[(size_t)i * V + v];
      const T zi = JAC ? mul(ri, c[i]) : z[(size_t)i * V + v];
      acc[v] += FLEX ? prod(zi, q[(size_t)i * V + v]) : prod(ri, zi);
    }
  }
  double tot[V];
  if (seg_commit<V>(sm, b, s, part, acc, tot) && threadIdx.x == 0) {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      Lane& L = lanes[s * V + v];
      if (!L.active) continue;
      if (FLEX) {
        L.beta = flex_beta(L, tot[v], c1 - c0);
        continue;
      }
      double beta = 1.0 / L.s;   // :44
      L.s_prev = L.s;
      L.s = tot[v];              // :47
      L.beta = beta * L.s;       // :50
    }
  }
}

// p = z + beta p  (solv_cg.f90:53).  FLEX: also s = p.r, so that the step
// alpha = (p.r)/(p.q) of k_cg_spmv makes the new residual orthogonal to p
// in the arithmetic actually done (flexible CG).
template <typename T, int V, bool JAC, bool FLEX = false>
__global__ void SG_BOUNDS(V) k_cg_p(SegMap sm, const T* __restrict__ c, const T* __restrict__ r,
                       const T* __restrict__ z, T* __restrict__ p,
                       Lane* __restrict__ lanes, double* __restrict__ part = nullptr) {
  const int b = blockIdx.x, s = sm.blk_seg[b];
  bool act[V];
  T beta[V];
  bool any = false;
#pragma unroll
  for (int v = 0; v < V; ++v) {
    act[v] = lanes[s * V + v].active != 0;
    beta[v] = (T)lanes[s * V + v].beta;
    any |= act[v];
  }
  if (!any) return;
  const int c0 = sm.seg_c0[s], c1 = sm.seg_c1[s];
  const int stride = sm.seg_nblk[s] * blockDim.x;
  double acc[V];
#pragma unroll
  for (int v = 0; v < V; ++v) acc[v] = 0.0;
  for (int i = c0 + sm.blk_rank[b] * blockDim.x + threadIdx.x; i < c1; i += stride) {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      if (!act[v]) continue;
      const size_t k = (size_t)i * V + v;
      const T ri = (JAC || FLEX) ? r[k] : T(0);
      const T zi = JAC ? mul(ri, c[i]) : z[k];
      const T pn = add(zi, mul(beta[v], p[k]));
      p[k] = pn;
      if (FLEX) acc[v] += prod(pn, ri);
    }
  }
  if constexpr (FLEX) {
    double tot[V];
    if (seg_commit<V>(sm, b, s, part, acc, tot) && threadIdx.x == 0) {
#pragma unroll
      for (int v = 0; v < V; ++v)
        if (act[v]) lanes[s * V + v].s = tot[v];
    }
  }
}

// q = A p and p.q; alpha = s / (p.q + small)   (solv_cg.f90:56-68; the FP32
// instantiation divides without the guard, div0)
template <typename T, int V, int CH = kRowChunk>
__global__ void SG_BOUNDS(V) k_cg_spmv(Rows<T> R, SegMap sm, const T* __restrict__ p, T* __restrict__ q,
                          double* __restrict__ part, Lane* __restrict__ lanes) {
  const int b = blockIdx.x, s = sm.blk_seg[b];
  bool any = false;
#pragma unroll
  for (int v = 0; v < V; ++v) any |= lanes[s * V + v].active != 0;
  if (!any) return;
  const int c0 = sm.seg_c0[s], c1 = sm.seg_c1[s];
  const int stride = sm.seg_nblk[s] * blockDim.x;
  double acc[V];
#pragma unroll
  for (int v = 0; v < V; ++v) acc[v] = 0.0;
  for (int i = c0 + sm.blk_rank[b] * blockDim.x + threadIdx.x; i < c1; i += stride) {
    T y[V];
    row_apply<T, V, CH>(R, i, p, y);
#pragma unroll
    for (int v = 0; v < V; ++v) {
      q[(size_t)i * V + v] = y[v];
      acc[v] += prod(p[(size_t)i * V + v], y[v]);
    }
  }
  double tot[V];
  if (seg_commit<V>(sm, b, s, part, acc, tot) && threadIdx.x == 0) {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      Lane& L = lanes[s * V + v];
      if (!L.active) continue;
      L.pq = tot[v];
      if constexpr (sizeof(T) == 4) L.alpha = div0(L.s, tot[v]);
      else L.alpha = L.s / (tot[v] + kSmall);  // :67-68
    }
  }
}

// phi += alpha p; r -= alpha q; L1 = sum|r|; stop test (solv_cg.f90:73-82).
// With JAC, also s_next = r.(c r) and beta for the next iteration; with
// JAC and FLEX, beta = -(z.q)/(p.q) instead, z = c r of the new residual.
template <typename T, int V, bool JAC, bool FLEX = false>
__global__ void SG_BOUNDS(V) k_cg_update(SegMap sm, const T* __restrict__ c, T* __restrict__ phi,
                            T* __restrict__ r, const T* __restrict__ p,
                            const T* __restrict__ q, double* __restrict__ part,
                            Lane* __restrict__ lanes) {
  const int b = blockIdx.x, s = sm.blk_seg[b];
  bool act[V];
  T alpha[V];
  bool any = false;
#pragma unroll
  for (int v = 0; v < V; ++v) {
    act[v] = lanes[s * V + v].active != 0;
    alpha[v] = (T)lanes[s * V + v].alpha;
    any |= act[v];
  }
  if (!any) return;
  const int c0 = sm.seg_c0[s], c1 = sm.seg_c1[s];
  const int stride = sm.seg_nblk[s] * blockDim.x;
  constexpr int NR = JAC ? 2 * V : V;
  double acc[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) acc[k] = 0.0;
  for (int i = c0 + sm.blk_rank[b] * blockDim.x + threadIdx.x; i < c1; i += stride) {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      if (!act[v]) continue;
      const size_t k = (size_t)i * V + v;
      phi[k] = add(phi[k], mul(alpha[v], p[k]));
      const T rn = sub(r[k], mul(alpha[v], q[k]));
      r[k] = rn;
      acc[v] += (double)fabs(rn);
      if (JAC) acc[V + v] += FLEX ? prod(mul(rn, c[i]), q[k]) : prod(rn, mul(rn, c[i]));
    }
  }
  double tot[NR];
  if (seg_commit<NR>(sm, b, s, part, acc, tot) && threadIdx.x == 0) {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      Lane& L = lanes[s * V + v];
      if (!L.active) continue;
      L.iter += 1;
      L.l1 = tot[v];
      const double ratio = tot[v] / (L.res0_n + kSmall);  // :81
      L.ratio = ratio;
      if (!(ratio == ratio) || isinf(ratio)) lane_stop(L, kLaneNaN, sm.n_active);
      else if (ratio < L.reduc) lane_stop(L, kLaneConverged, sm.n_active);  // :82
      else if (L.iter >= L.n_iter) lane_stop(L, kLaneMaxIter, sm.n_active);
      else if (tot[v] < L.l1_stop) lane_stop(L, kLaneRefine, sm.n_active);
      if (JAC && FLEX && L.active) {
        L.beta = flex_beta(L, tot[V + v], c1 - c0);
      } else if (JAC && L.active) {
        double beta = 1.0 / L.s;
        L.s_prev = L.s;
        L.s = tot[V + v];
        L.beta = beta * L.s;
      }
    }
  }
}

// ===================== BiCGSTAB: solv_bicg.f90:27-118 ======================
// rho = r.r0; omeg = rho*gam/(alpha*beta0+small); beta0 = rho  (:48-50;
// FP32 without the guard, div0)
template <typename T, int V>
__global__ void SG_BOUNDS(V) k_bi_rho(SegMap sm, const T* __restrict__ r, const T* __restrict__ r0,
                         double* __restrict__ part, Lane* __restrict__ lanes) {
  const int b = blockIdx.x, s = sm.blk_seg[b];
  bool any = false;
#pragma unroll
  for (int v = 0; v < V; ++v) any |= lanes[s * V + v].active != 0;
  if (!any) return;
  const int c0 = sm.seg_c0[s], c1 = sm.seg_c1[s];
  const int stride = sm.seg_nblk[s] * blockDim.x;
  double acc[V];
#pragma unroll
  for (int v = 0; v < V; ++v) acc[v] = 0.0;
  for (int i = c0 + sm.blk_rank[b] * blockDim.x + threadIdx.x; i < c1; i += stride) {
#pragma unroll
    for (int v = 0; v < V; ++v) acc[v] += prod(r[(size_t)i * V + v], r0[(size_t)i * V + v]);
  }
  double tot[V];
  if (seg_commit<V>(sm, b, s, part, acc, tot) && threadIdx.x == 0) {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      Lane& L = lanes[s * V + v];
      if (!L.active) continue;
      L.rho = tot[v];
      if constexpr (sizeof(T) == 4) L.omeg = div0(L.rho * L.gam, L.alpha * L.beta0);
      else L.omeg = L.rho * L.gam / (L.alpha * L.beta0 + kSmall);
      L.beta0 = L.rho;
    }
  }
}

// p = r + omeg (p - alpha u); with JAC also z = c p  (:54-58)
template <typename T, int V, bool JAC>
__global__ void SG_BOUNDS(V) k_bi_p(SegMap sm, const T* __restrict__ c, const T* __restrict__ r,
                       T* __restrict__ p, const T* __restrict__ u, T* __restrict__ z,
                       const Lane* __restrict__ lanes) {
  const int b = blockIdx.x, s = sm.blk_seg[b];
  bool act[V];
  T om[V], al[V];
  bool any = false;
#pragma unroll
  for (int v = 0; v < V; ++v) {
    act[v] = lanes[s * V + v].active != 0;
    om[v] = (T)lanes[s * V + v].omeg;
    al[v] = (T)lanes[s * V + v].alpha;
    any |= act[v];
  }
  if (!any) return;
  const int c0 = sm.seg_c0[s], c1 = sm.seg_c1[s];
  const int stride = sm.seg_nblk[s] * blockDim.x;
  for (int i = c0 + sm.blk_rank[b] * blockDim.x + threadIdx.x; i < c1; i += stride) {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      if (!act[v]) continue;
      const size_t k = (size_t)i * V + v;
      const T pn = add(r[k], mul(om[v], sub(p[k], mul(al[v], u[k]))));
      p[k] = pn;
      if (JAC) z[k] = mul(pn, c[i]);
    }
  }
}

// y = A z, and dots: MODE 0 -> y.r0 (gam = rho/(y.r0+small), :72-73)
//                    MODE 1 -> y.r, y.y (alpha = (y.r)/(y.y+small), :98-100)
// (FP32: the same quotients without the guard, div0)
template <typename T, int V, int MODE, int CH = kRowChunk>
__global__ void SG_BOUNDS(V) k_bi_spmv(Rows<T> R, SegMap sm, const T* __restrict__ z, T* __restrict__ y,
                          const T* __restrict__ w, double* __restrict__ part,
                          Lane* __restrict__ lanes) {
  const int b = blockIdx.x, s = sm.blk_seg[b];
  bool any = false;
#pragma unroll
  for (int v = 0; v < V; ++v) any |= lanes[s * V + v].active != 0;
  if (!any) return;
  const int c0 = sm.seg_c0[s], c1 = sm.seg_c1[s];
  const int stride = sm.seg_nblk[s] * blockDim.x;
  constexpr int NR = MODE == 0 ? V : 2 * V;
  double acc[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) acc[k] = 0.0;
  for (int i = c0 + sm.blk_rank[b] * blockDim.x + threadIdx.x; i < c1; i += stride) {
    T t[V];
    row_apply<T, V, CH>(R, i, z, t);
#pragma unroll
    for (int v = 0; v < V; ++v) {
      y[(size_t)i * V + v] = t[v];
      acc[v] += prod(t[v], w[(size_t)i * V + v]);
      if (MODE == 1) acc[V + v] += prod(t[v], t[v]);
    }
  }
  double tot[NR];
  if (seg_commit<NR>(sm, b, s, part, acc, tot) && threadIdx.x == 0) {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      Lane& L = lanes[s * V + v];
      if (!L.active) continue;
      if (MODE == 0) {
        if constexpr (sizeof(T) == 4) L.gam = div0(L.rho, tot[v]);
        else L.gam = L.rho / (tot[v] + kSmall);
      } else {
        if constexpr (sizeof(T) == 4) L.alpha = div0(tot[v], tot[V + v]);
        else L.alpha = tot[v] / (tot[V + v] + kSmall);
      }
    }
  }
}

// phi += gam z; r -= gam u; with JAC also z = c r   (:77-84)
template <typename T, int V, bool JAC>
__global__ void SG_BOUNDS(V) k_bi_half(SegMap sm, const T* __restrict__ c, T* __restrict__ phi,
                          T* __restrict__ r, T* __restrict__ z, const T* __restrict__ u,
                          const Lane* __restrict__ lanes) {
  const int b = blockIdx.x, s = sm.blk_seg[b];
  bool act[V];
  T g[V];
  bool any = false;
#pragma unroll
  for (int v = 0; v < V; ++v) {
    act[v] = lanes[s * V + v].active != 0;
    g[v] = (T)lanes[s * V + v].gam;
    any |= act[v];
  }
  if (!any) return;
  const int c0 = sm.seg_c0[s], c1 = sm.seg_c1[s];
  const int stride = sm.seg_nblk[s] * blockDim.x;
  for (int i = c0 + sm.blk_rank[b] * blockDim.x + threadIdx.x; i < c1; i += stride) {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      if (!act[v]) continue;
      const size_t k = (size_t)i * V + v;
      phi[k] = add(phi[k], mul(g[v], z[k]));
      const T rn = sub(r[k], mul(g[v], u[k]));
      r[k] = rn;
      if (JAC) z[k] = mul(rn, c[i]);
    }
  }
}

// phi += alpha z; r -= alpha v; L1; stop test; rho_next = r.r0 with the
// omeg / beta0 update of the next iteration's head (:105-116, :48-50).
template <typename T, int V>
__global__ void SG_BOUNDS(V) k_bi_update(SegMap sm, T* __restrict__ phi, T* __restrict__ r,
                            const T* __restrict__ z, const T* __restrict__ vv,
                            const T* __restrict__ r0, double* __restrict__ part,
                            Lane* __restrict__ lanes) {
  const int b = blockIdx.x, s = sm.blk_seg[b];
  bool act[V];
  T al[V];
  bool any = false;
#pragma unroll
  for (int v = 0; v < V; ++v) {
    act[v] = lanes[s * V + v].active != 0;
    al[v] = (T)lanes[s * V + v].alpha;
    any |= act[v];
  }
  if (!any) return;
  const int c0 = sm.seg_c0[s], c1 = sm.seg_c1[s];
  const int stride = sm.seg_nblk[s] * blockDim.x;
  double acc[2 * V];
#pragma unroll
  for (int k = 0; k < 2 * V; ++k) acc[k] = 0.0;
  for (int i = c0 + sm.blk_rank[b] * blockDim.x + threadIdx.x; i < c1; i += stride) {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      if (!act[v]) continue;
      const size_t k = (size_t)i * V + v;
      phi[k] = add(phi[k], mul(al[v], z[k]));
      const T rn = sub(r[k], mul(al[v], vv[k]));
      r[k] = rn;
      acc[v] += (double)fabs(rn);
      acc[V + v] += prod(rn, r0[k]);
    }
  }
  double tot[2 * V];
  if (seg_commit<2 * V>(sm, b, s, part, acc, tot) && threadIdx.x == 0) {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      Lane& L = lanes[s * V + v];
      if (!L.active) continue;
      L.iter += 1;
      L.l1 = tot[v];
      const double ratio = tot[v] / (L.res0_n + kSmall);
      L.ratio = ratio;
      if (!(ratio == ratio) || isinf(ratio)) lane_stop(L, kLaneNaN, sm.n_active);
      else if (ratio < L.reduc) lane_stop(L, kLaneConverged, sm.n_active);
      else if (L.iter >= L.n_iter) lane_stop(L, kLaneMaxIter, sm.n_active);
      else if (tot[v] < L.l1_stop) lane_stop(L, kLaneRefine, sm.n_active);
      if (L.active) {
        L.rho = tot[V + v];
        if constexpr (sizeof(T) == 4) L.omeg = div0(L.rho * L.gam, L.alpha * L.beta0);
        else L.omeg = L.rho * L.gam / (L.alpha * L.beta0 + kSmall);
        L.beta0 = L.rho;
      }
    }
  }
}

// ================ reliable updates for the mixed-precision CG =================
// d (FP32 correction since the last update) -> x (FP64) for every lane
// flagged in mask, and d = 0.
template <int V>
__global__ void SG_BOUNDS(V) k_mp_flush(SegMap sm, const int* __restrict__ mask, double* __restrict__ x,
                           float* __restrict__ d) {
  const int b = blockIdx.x, s = sm.blk_seg[b];
  bool on[V];
  bool any = false;
#pragma unroll
  for (int v = 0; v < V; ++v) { on[v] = mask[s * V + v] != 0; any |= on[v]; }
  if (!any) return;
  const int c0 = sm.seg_c0[s], c1 = sm.seg_c1[s];
  const int stride = sm.seg_nblk[s] * blockDim.x;
  for (int i = c0 + sm.blk_rank[b] * blockDim.x + threadIdx.x; i < c1; i += stride) {
#pragma unroll
    for (int v = 0; v < V; ++v)
      if (on[v]) {
        const size_t k = (size_t)i * V + v;
        x[k] += (double)d[k];
        d[k] = 0.0f;
      }
  }
}

// r_f = (float) r for the lanes in mask
template <int V>
__global__ void SG_BOUNDS(V) k_mp_replace(SegMap sm, const int* __restrict__ mask, const double* __restrict__ r,
                             float* __restrict__ rf) {
  const int b = blockIdx.x, s = sm.blk_seg[b];
  bool on[V];
  bool any = false;
#pragma unroll
  for (int v = 0; v < V; ++v) { on[v] = mask[s * V + v] != 0; any |= on[v]; }
  if (!any) return;
  const int c0 = sm.seg_c0[s], c1 = sm.seg_c1[s];
  const int stride = sm.seg_nblk[s] * blockDim.x;
  for (int i = c0 + sm.blk_rank[b] * blockDim.x + threadIdx.x; i < c1; i += stride) {
#pragma unroll
    for (int v = 0; v < V; ++v)
      if (on[v]) rf[(size_t)i * V + v] = (float)r[(size_t)i * V + v];
  }
}

// ================ flexible CG, FCG(1), for a nonlinear preconditioner ==========
// z = M(r); beta = -(z.q_old)/(p_old.q_old); p = z + beta p; q = A p;
// alpha = (p.r)/(p.q); x += alpha p; r -= alpha q.  One system, V = 1.

// gs = sum |r_i| rsd_i / N: the residual scale the network normalises by.
template <typename T>
__global__ void SG_BOUNDS(1) k_fcg_scale(SegMap sm, const T* __restrict__ r, const float* __restrict__ rsd,
                            double* __restrict__ part, Lane* __restrict__ lanes) {
  const int b = blockIdx.x, s = sm.blk_seg[b];
  if (!lanes[s].active) return;
  const int c0 = sm.seg_c0[s], c1 = sm.seg_c1[s];
  const int stride = sm.seg_nblk[s] * blockDim.x;
  double acc[1] = {0.0};
  for (int i = c0 + sm.blk_rank[b] * blockDim.x + threadIdx.x; i < c1; i += stride)
    acc[0] += fabs((double)r[i]) * rsd[i];
  double tot[1];
  if (seg_commit<1>(sm, b, s, part, acc, tot) && threadIdx.x == 0)
    lanes[s].gs = tot[0] / (double)(c1 - c0);
}

template <typename T>
__global__ void SG_BOUNDS(1) k_fcg_beta(SegMap sm, const T* __restrict__ z, const T* __restrict__ q,
                           double* __restrict__ part, Lane* __restrict__ lanes) {
  const int b = blockIdx.x, s = sm.blk_seg[b];
  if (!lanes[s].active) return;
  const int c0 = sm.seg_c0[s], c1 = sm.seg_c1[s];
  const int stride = sm.seg_nblk[s] * blockDim.x;
  double acc[1] = {0.0};
  for (int i = c0 + sm.blk_rank[b] * blockDim.x + threadIdx.x; i < c1; i += stride)
    acc[0] += prod(z[i], q[i]);
  double tot[1];
  if (seg_commit<1>(sm, b, s, part, acc, tot) && threadIdx.x == 0) {
    Lane& L = lanes[s];
    L.beta = flex_beta(L, tot[0], c1 - c0);
  }
}

template <typename T, int CH = kRowChunk>
__global__ void SG_BOUNDS(1) k_fcg_spmv(Rows<T> R, SegMap sm, const T* __restrict__ p, T* __restrict__ q,
                           const T* __restrict__ r, double* __restrict__ part,
                           Lane* __restrict__ lanes) {
  const int b = blockIdx.x, s = sm.blk_seg[b];
  if (!lanes[s].active) return;
  const int c0 = sm.seg_c0[s], c1 = sm.seg_c1[s];
  const int stride = sm.seg_nblk[s] * blockDim.x;
  double acc[2] = {0.0, 0.0};
  for (int i = c0 + sm.blk_rank[b] * blockDim.x + threadIdx.x; i < c1; i += stride) {
    T y[1];
    row_apply<T, 1, CH>(R, i, p, y);
    q[i] = y[0];
    acc[0] += prod(p[i], y[0]);
    acc[1] += prod(p[i], r[i]);
  }
  double tot[2];
  if (seg_commit<2>(sm, b, s, part, acc, tot) && threadIdx.x == 0) {
    Lane& L = lanes[s];
    if (!(tot[0] > 0.0) || !(tot[1] == tot[1])) {  // not SPD-like: hand over to PCG
      L.alpha = 0.0;
      lane_stop(L, kLaneStall, sm.n_active);
    } else {
      L.pq = tot[0];
      L.alpha = tot[1] / tot[0];
    }
  }
}

template <typename T>
__global__ void SG_BOUNDS(1) k_fcg_update(SegMap sm, T* __restrict__ phi, T* __restrict__ r,
                             const T* __restrict__ p, const T* __restrict__ q,
                             double* __restrict__ part, Lane* __restrict__ lanes) {
  const int b = blockIdx.x, s = sm.blk_seg[b];
  if (!lanes[s].active) return;
  const T alpha = (T)lanes[s].alpha;
  const int c0 = sm.seg_c0[s], c1 = sm.seg_c1[s];
  const int stride = sm.seg_nblk[s] * blockDim.x;
  double acc[1] = {0.0};
  for (int i = c0 + sm.blk_rank[b] * blockDim.x + threadIdx.x; i < c1; i += stride) {
    phi[i] = add(phi[i], mul(alpha, p[i]));
    const T rn = sub(r[i], mul(alpha, q[i]));
    r[i] = rn;
    acc[0] += fabs((double)rn);
  }
  double tot[1];
  if (seg_commit<1>(sm, b, s, part, acc, tot) && threadIdx.x == 0) {
    Lane& L = lanes[s];
    L.iter += 1;
    L.l1 = tot[0];
    const double ratio = tot[0] / (L.res0_n + kSmall);
    L.ratio = ratio;
    if (!(ratio == ratio) || isinf(ratio)) lane_stop(L, kLaneNaN, sm.n_active);
    else if (ratio < L.reduc) lane_stop(L, kLaneConverged, sm.n_active);
    else if (L.iter >= L.n_iter) lane_stop(L, kLaneMaxIter, sm.n_active);
    else if (tot[0] < L.l1_stop) lane_stop(L, kLaneRefine, sm.n_active);
  }
}

// ============ persistent fused Jacobi PCG: one thread-block cluster per system ============
// The whole Krylov loop of solv_cg.f90:37-84 with imat = 0 in one launch:
// each cluster of CTAs (kPcgCluster, or kPcgClusterMax where the GPU holds
// a cluster that large at once) owns one system (segment) and iterates it
// to its stopping test, fusing the Jacobi step into the direction update,
// the product with p.q, and the solution / residual update with |r|_1 and
// r.z.  Per iteration three cluster barriers (after p; after the p.q
// partials; after the update's partials); each CTA reduces its cells in a
// fixed tree, puts its partials in shared memory, and in every CTA one warp
// reads the cluster's partials over distributed shared memory (a lane per
// rank) and sums them in a fixed tree -- so all CTAs hold the same scalars
// and take the same branch, and the sums are deterministic.  Per-cell arithmetic is the graph path's (k_cg_p,
// k_cg_spmv, k_cg_update with JAC), so a solve differs from it only in the
// reduction trees.  The loop is bounded by the lane's n_iter.
constexpr int kPcgCluster = 8;      // portable cluster size
constexpr int kPcgClusterMax = 16;  // non-portable, one system's whole GPC
constexpr int kPcgThreads = 1024;

__device__ __forceinline__ double cluster_block_sum(double v, double* red) {
  // fixed-order block sum; result in every thread
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  v = warp_sum(v);
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (w == 0) {
    t = l < (int)(blockDim.x >> 5) ? red[l] : 0.0;
    t = warp_sum(t);
    if (l == 0) red[32] = t;
  }
  __syncthreads();
  return red[32];
}

// Two fixed-order block sums in one pass (red holds 2 x 33 doubles).
__device__ __forceinline__ void cluster_block_sum2(double& a, double& b, double* red) {
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  a = warp_sum(a);
  b = warp_sum(b);
  __syncthreads();
  if (l == 0) {
    red[w] = a;
    red[33 + w] = b;
  }
  __syncthreads();
  if (w == 0) {
    const bool in = l < (int)(blockDim.x >> 5);
    double ta = warp_sum(in ? red[l] : 0.0);
    double tb = warp_sum(in ? red[33 + l] : 0.0);
    if (l == 0) {
      red[32] = ta;
      red[65] = tb;
    }
  }
  __syncthreads();
  a = red[32];
  b = red[65];
}

// y_i = (A p)_i for two rows at once (i1 < 0: none), each summed in slot
// order as row_apply does; slot k of both rows is loaded before either is
// added, so two independent gathers are in flight (two slots a row spilled
// under the 64 registers a 1024-thread block allows).
__device__ __forceinline__ void row_pair_apply(const Rows<double>& R, int i0, int i1,
                                               const double* p, double& y0, double& y1) {
  RowIt<double> r0(R, i0);
  RowIt<double> r1(R, i1 >= 0 ? i1 : i0);
  const int w0 = r0.w, w1 = i1 >= 0 ? r1.w : 0;
  y0 = mul(R.diag[i0], __ldcg(&p[i0]));
  y1 = i1 >= 0 ? mul(R.diag[i1], __ldcg(&p[i1])) : 0.0;
  const int wm = max(w0, w1);
  for (int k = 0; k < wm; ++k) {
    int j0 = -1, j1 = -1;
    double a0 = 0.0, a1 = 0.0;
    if (k < w0) {
      const int e = r0.base + k * kWarp;
      j0 = __ldg(&R.col[e]);
      a0 = __ldg(&R.val[e]);
    }
    if (k < w1) {
      const int e = r1.base + k * kWarp;
      j1 = __ldg(&R.col[e]);
      a1 = __ldg(&R.val[e]);
    }
    const double x0 = j0 >= 0 ? __ldcg(&p[j0]) : 0.0;
    const double x1 = j1 >= 0 ? __ldcg(&p[j1]) : 0.0;
    if (j0 >= 0) y0 = add(y0, mul(a0, x0));
    if (j1 >= 0) y1 = add(y1, mul(a1, x1));
  }
}

__global__ void __launch_bounds__(kPcgThreads) k_pcg_cluster(
    Rows<double> R, const int* __restrict__ seg_c0, const int* __restrict__ seg_c1,
    const double* __restrict__ c, double* __restrict__ phi, double* __restrict__ r,
    double* __restrict__ p, double* __restrict__ q, Lane* __restrict__ lanes,
    int* __restrict__ n_active) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  __shared__ double red[66];
  __shared__ double part[2][2];  // this CTA's partials: [product][update]
  __shared__ double tot_s[2];
  const int rank = (int)cl.block_rank(), cs = (int)cl.num_blocks();
  const int sys = blockIdx.x / cs;
  const int c0 = seg_c0[sys], c1 = seg_c1[sys];
  const int stride = cs * blockDim.x;
  const int first = c0 + rank * blockDim.x + threadIdx.x;
  // the lane's scalars, in registers (the Lane itself is written back once)
  const Lane L0 = lanes[sys];
  if (!L0.active) return;  // uniform over the cluster
  const double res0_n = L0.res0_n, reduc = L0.reduc;
  const int n_iter = L0.n_iter;
  double s_cur = L0.s, s_prev = L0.s_prev, beta = 0.0, alpha = L0.alpha, pq = L0.pq;
  double l1v = L0.l1, ratio = L0.ratio;
  int iter = L0.iter;
  // the cluster's totals of one partial slot: lane q of warp 0 reads rank
  // q's pair over distributed shared memory, the warp sums them in a fixed
  // tree (the same in every CTA), and the block takes the pair from there
  auto cluster_totals = [&](int slot, double& t0, double& t1) {
    if (threadIdx.x < 32) {
      const int l = threadIdx.x;
      double a = 0.0, b = 0.0;
      if (l < cs) {
        const double* pp = cl.map_shared_rank(&part[slot][0], l);
        a = pp[0];
        b = pp[1];
      }
      a = warp_sum(a);
      b = warp_sum(b);
      if (l == 0) {
        tot_s[0] = a;
        tot_s[1] = b;
      }
    }
    __syncthreads();
    t0 = tot_s[0];
    t1 = tot_s[1];
  };
  // s = r.(c r), beta = (1/s_old) s (k_cg_rz with JAC)
  {
    double a = 0.0;
    for (int i = first; i < c1; i += stride) {
      const double ri = r[i];
      a += prod(ri, mul(ri, c[i]));
    }
    a = cluster_block_sum(a, red);
    if (threadIdx.x == 0) {
      part[1][0] = a;
      part[1][1] = 0.0;
    }
    cl.sync();
    double s_new, unused;
    cluster_totals(1, s_new, unused);
    const double b0 = 1.0 / s_cur;
    s_prev = s_cur;
    s_cur = s_new;
    beta = b0 * s_cur;
  }
  int status = kLaneRunning;
  while (true) {
    // (a partial slot is rewritten only two barriers after its last read)
    // p = z + beta p, z = c r (k_cg_p with JAC)
    for (int i = first; i < c1; i += stride) {
      const double zi = mul(r[i], c[i]);
      p[i] = add(zi, mul(beta, p[i]));
    }
    cl.sync();  // p complete in the cluster
    // q = A p, p.q (k_cg_spmv); neighbours' p read past L1; two rows at a time
    double a = 0.0;
    for (int i = first; i < c1; i += 2 * stride) {
      const int i1 = i + stride < c1 ? i + stride : -1;
      double y0, y1;
      row_pair_apply(R, i, i1, p, y0, y1);
      q[i] = y0;
      a += prod(__ldcg(&p[i]), y0);
      if (i1 >= 0) {
        q[i1] = y1;
        a += prod(__ldcg(&p[i1]), y1);
      }
    }
    a = cluster_block_sum(a, red);
    if (threadIdx.x == 0) {
      part[0][0] = a;
      part[0][1] = 0.0;
    }
    cl.sync();
    double unused2;
    cluster_totals(0, pq, unused2);
    alpha = s_cur / (pq + kSmall);  // solv_cg.f90:67-68
    // phi += alpha p; r -= alpha q; |r|_1; r.(c r) (k_cg_update with JAC)
    double l1 = 0.0, rz = 0.0;
    for (int i = first; i < c1; i += stride) {
      phi[i] = add(phi[i], mul(alpha, p[i]));
      const double rn = sub(r[i], mul(alpha, q[i]));
      r[i] = rn;
      l1 += fabs(rn);
      rz += prod(rn, mul(rn, c[i]));
    }
    cluster_block_sum2(l1, rz, red);
    if (threadIdx.x == 0) {
      part[1][0] = l1;
      part[1][1] = rz;
    }
    cl.sync();
    double t1, t2;
    cluster_totals(1, t1, t2);
    iter += 1;
    l1v = t1;
    ratio = t1 / (res0_n + kSmall);  // solv_cg.f90:81
    if (!(ratio == ratio) || isinf(ratio)) status = kLaneNaN;
    else if (ratio < reduc) status = kLaneConverged;  // :82
    else if (iter >= n_iter) status = kLaneMaxIter;
    if (status != kLaneRunning) break;
    const double b1 = 1.0 / s_cur;
    s_prev = s_cur;
    s_cur = t2;
    beta = b1 * s_cur;
  }
  cl.sync();  // no CTA leaves while others may still read its partials
  if (rank == 0 && threadIdx.x == 0) {
    Lane L = L0;
    L.s = s_cur;
    L.s_prev = s_prev;
    L.beta = beta;
    L.alpha = alpha;
    L.pq = pq;
    L.iter = iter;
    L.l1 = l1v;
    L.ratio = ratio;
    L.active = 0;
    L.status = status;
    lanes[sys] = L;
    atomicSub(n_active, 1);
  }
}

// The same loop for a system small enough for one cluster to hold
// (at most cs x 1024 x RPT cells): each CTA owns a contiguous block of
// B = 1024 x RPT cells, keeps their r, c, phi, p and q in registers (RPT
// cells a thread) and their p in shared memory, and the product reads a
// neighbour's p over distributed shared memory from the CTA that owns it
// -- no vector goes through L2 inside the loop, only the matrix slots
// (read-only, L1-resident after the first pass).  Per-cell arithmetic and
// the slot order of the sums are the global-memory kernel's.
template <int RPT>
__global__ void __launch_bounds__(kPcgThreads) k_pcg_cluster_res(
    Rows<double> R, const int* __restrict__ seg_c0, const int* __restrict__ seg_c1,
    const double* __restrict__ c, double* __restrict__ phi, double* __restrict__ r,
    double* __restrict__ p, double* __restrict__ q, Lane* __restrict__ lanes,
    int* __restrict__ n_active) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  constexpr int B = kPcgThreads * RPT;
  constexpr int LOGB = RPT == 1 ? 10 : 11;
  static_assert(RPT == 1 || RPT == 2, "one or two cells a thread");
  __shared__ double p_s[B];
  __shared__ double red[66];
  __shared__ double part[2][2];
  __shared__ double tot_s[2];
  const int rank = (int)cl.block_rank(), cs = (int)cl.num_blocks();
  const int sys = blockIdx.x / cs;
  const int c0 = seg_c0[sys], c1 = seg_c1[sys];
  const Lane L0 = lanes[sys];
  if (!L0.active) return;  // uniform over the cluster
  int row[RPT];
  double rr[RPT], cc[RPT], ph[RPT], pp[RPT], qq[RPT];
#pragma unroll
  for (int u = 0; u < RPT; ++u) {
    row[u] = c0 + rank * B + u * kPcgThreads + (int)threadIdx.x;
    const bool h = row[u] < c1;
    rr[u] = h ? r[row[u]] : 0.0;
    cc[u] = h ? c[row[u]] : 0.0;
    ph[u] = h ? phi[row[u]] : 0.0;
    pp[u] = h ? p[row[u]] : 0.0;
    qq[u] = 0.0;
    if (!h) row[u] = -1;
  }
  const double res0_n = L0.res0_n, reduc = L0.reduc;
  const int n_iter = L0.n_iter;
  double s_cur = L0.s, s_prev = L0.s_prev, beta = 0.0, alpha = L0.alpha, pq = L0.pq;
  double l1v = L0.l1, ratio = L0.ratio;
  int iter = L0.iter;
  auto cluster_totals = [&](int slot, double& t0, double& t1) {
    if (threadIdx.x < 32) {
      const int l = threadIdx.x;
      double a = 0.0, b = 0.0;
      if (l < cs) {
        const double* pr = cl.map_shared_rank(&part[slot][0], l);
        a = pr[0];
        b = pr[1];
      }
      a = warp_sum(a);
      b = warp_sum(b);
      if (l == 0) {
        tot_s[0] = a;
        tot_s[1] = b;
      }
    }
    __syncthreads();
    t0 = tot_s[0];
    t1 = tot_s[1];
  };
  // s = r.(c r), beta = (1/s_old) s
  {
    double a = 0.0;
#pragma unroll
    for (int u = 0; u < RPT; ++u)
      if (row[u] >= 0) a += prod(rr[u], mul(rr[u], cc[u]));
    a = cluster_block_sum(a, red);
    if (threadIdx.x == 0) {
      part[1][0] = a;
      part[1][1] = 0.0;
    }
    cl.sync();
    double s_new, unused;
    cluster_totals(1, s_new, unused);
    const double b0 = 1.0 / s_cur;
    s_prev = s_cur;
    s_cur = s_new;
    beta = b0 * s_cur;
  }
  int status = kLaneRunning;
  while (true) {
    // p = z + beta p, z = c r; this CTA's p into shared memory
#pragma unroll
    for (int u = 0; u < RPT; ++u) {
      if (row[u] >= 0) pp[u] = add(mul(rr[u], cc[u]), mul(beta, pp[u]));
      p_s[u * kPcgThreads + threadIdx.x] = pp[u];
    }
    cl.sync();  // every CTA's p visible in the cluster
    // q = A p, p.q: neighbours' p from their owners' shared memory
    double a = 0.0;
#pragma unroll
    for (int u = 0; u < RPT; ++u) {
      if (row[u] < 0) continue;
      RowIt<double> it(R, row[u]);
      double y = mul(__ldg(&R.diag[row[u]]), pp[u]);
      for (int k0 = 0; k0 < it.w; k0 += 4) {
        int j[4];
        double av[4], xv[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          j[v] = -1;
          av[v] = 0.0;
          if (k0 + v < it.w) {
            const int e = it.base + (k0 + v) * kWarp;
            j[v] = __ldg(&R.col[e]);
            av[v] = __ldg(&R.val[e]);
          }
        }
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          xv[v] = 0.0;
          if (j[v] >= 0) {
            const int o = j[v] - c0;
            xv[v] = *cl.map_shared_rank(&p_s[o & (B - 1)], o >> LOGB);
          }
        }
#pragma unroll
        for (int v = 0; v < 4; ++v)
          if (j[v] >= 0) y = add(y, mul(av[v], xv[v]));
      }
      qq[u] = y;
      a += prod(pp[u], y);
    }
    a = cluster_block_sum(a, red);
    if (threadIdx.x == 0) {
      part[0][0] = a;
      part[0][1] = 0.0;
    }
    cl.sync();
    double unused2;
    cluster_totals(0, pq, unused2);
    alpha = s_cur / (pq + kSmall);  // solv_cg.f90:67-68
    double l1 = 0.0, rz = 0.0;
#pragma unroll
    for (int u = 0; u < RPT; ++u) {
      if (row[u] < 0) continue;
      ph[u] = add(ph[u], mul(alpha, pp[u]));
      const double rn = sub(rr[u], mul(alpha, qq[u]));
      rr[u] = rn;
      l1 += fabs(rn);
      rz += prod(rn, mul(rn, cc[u]));
    }
    cluster_block_sum2(l1, rz, red);
    if (threadIdx.x == 0) {
      part[1][0] = l1;
      part[1][1] = rz;
    }
    cl.sync();
    double t1, t2;
    cluster_totals(1, t1, t2);
    iter += 1;
    l1v = t1;
    ratio = t1 / (res0_n + kSmall);  // solv_cg.f90:81
    if (!(ratio == ratio) || isinf(ratio)) status = kLaneNaN;
    else if (ratio < reduc) status = kLaneConverged;  // :82
    else if (iter >= n_iter) status = kLaneMaxIter;
    if (status != kLaneRunning) break;
    const double b1 = 1.0 / s_cur;
    s_prev = s_cur;
    s_cur = t2;
    beta = b1 * s_cur;
  }
#pragma unroll
  for (int u = 0; u < RPT; ++u) {
    if (row[u] < 0) continue;
    phi[row[u]] = ph[u];
    r[row[u]] = rr[u];
    p[row[u]] = pp[u];
    q[row[u]] = qq[u];
  }
  cl.sync();  // no CTA leaves while others may still read its shared memory
  if (rank == 0 && threadIdx.x == 0) {
    Lane L = L0;
    L.s = s_cur;
    L.s_prev = s_prev;
    L.beta = beta;
    L.alpha = alpha;
    L.pq = pq;
    L.iter = iter;
    L.l1 = l1v;
    L.ratio = ratio;
    L.active = 0;
    L.status = status;
    lanes[sys] = L;
    atomicSub(n_active, 1);
  }
}

// How local a structure is for k_pcg_cluster_res: over all slots, how many
// have their neighbour in the same block of 2^logb cells of the system as
// the row (cnt[0] slots, cnt[1] local ones).  seg_c0/seg_c1 are sorted.
__global__ void k_block_locality(int n, Rows<double> R, const int* __restrict__ seg_c0,
                                 const int* __restrict__ seg_c1, int n_seg, int logb,
                                 unsigned long long* __restrict__ cnt) {
  unsigned long long tot = 0, loc = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int lo = 0, hi = n_seg - 1;  // the system of row i
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (seg_c0[mid] <= i) lo = mid;
      else hi = mid - 1;
    }
    const int c0 = seg_c0[lo];
    RowIt<double> it(R, i);
    for (int k = 0; k < it.w; ++k) {
      const int j = R.col[it.base + k * kWarp];
      if (j < 0) continue;
      ++tot;
      loc += ((j - c0) >> logb) == ((i - c0) >> logb);
    }
  }
  tot = (unsigned long long)warp_sum((double)tot);
  loc = (unsigned long long)warp_sum((double)loc);
  if ((threadIdx.x & 31) == 0 && tot) {
    atomicAdd(&cnt[0], tot);
    atomicAdd(&cnt[1], loc);
  }
}

// Loop control of a WHILE graph of Krylov iterations: one pass per
// iteration, on until every lane has stopped or the budget is spent.
__global__ void k_loop_ctl(cudaGraphConditionalHandle h, const int* __restrict__ n_active,
                           int* __restrict__ budget) {
  if (threadIdx.x == 0) {
    const int b = *budget - 1;
    *budget = b;
    cudaGraphSetConditional(h, (b > 0 && *n_active > 0) ? 1u : 0u);
  }
}

// Self-test of the recurrences' bounded wait: one slice whose only cell
// waits on a value nothing ever writes, through the same driver
// (sweep_slices) as the sweeps, so the wait runs out after kSweepPolls
// polls and sets ctl->err.  slice_w holds {1}; never is pending.
__global__ void k_sweep_selftest(const uint8_t* __restrict__ slice_w, const double* never,
                                 SweepCtl* ctl) {
  sweep_slices<false>(1, slice_w, ctl, [&](int i, int k, bool first) -> int {
    double v;
    return i == 0 && take(never, v) ? 1 : (i == 0 ? 0 : 1);
  });
}

}  // namespace sg
