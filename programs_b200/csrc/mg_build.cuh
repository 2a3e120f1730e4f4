// mg_build.cuh -- the aggregation hierarchy of mg.cuh, built on the GPU.
//
// One level of coarsening, from a level's sliced-ELL structure and its
// coupling strengths |a_ij| (FP32), all in device memory:
//
//   1. three passes of pairwise matching.  Each pass is a handshake: every
//      cell still free proposes to its most strongly coupled free neighbour
//      (ties: the lower index), and two cells that propose to each other
//      pair up; kRounds such rounds, then a cell left over joins the pair of
//      its most strongly coupled matched neighbour (on dense coarse graphs
//      proposals often form cycles and leave many cells unmatched; joined,
//      they still coarsen).  Aggregates are numbered by their lower pair
//      member (a prefix sum over the cells), which keeps the locality of
//      the level's numbering.  Passes 2
//      and 3 match the pass graphs: the aggregates so far, coupled by the
//      summed strengths of the couplings between them;
//   2. a cell left alone by all passes joins the aggregate of its most
//      strongly coupled neighbour that has more than one member (on the
//      level's own graph), and the aggregates are renumbered densely in
//      the order of their numbers;
//   3. the Galerkin structure of the coarse level: coarse row I lists the
//      aggregates J != I that I's members couple to, in order of first
//      appearance over I's members (ascending) and their slots, and coarse
//      slot (I, J) lists the finer slots that sum into it, in that order.
//      One warp per coarse row keeps the row's list in shared memory.
//
// Everything is deterministic: handshakes, counts and prefix sums do not
// depend on the scheduling, member lists are sorted, and the Galerkin walk
// visits every row's finer slots in a fixed order.  The structure it gives
// is the one mg.cuh's host build describes (same slot order rule), over a
// matching found in parallel instead of by a sequential greedy sweep.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.cuh"

namespace mgb {

constexpr int kRounds = 6;        // handshake rounds per matching pass
constexpr int kMaxRow = 255;      // coarse row width limit (8-bit slot counts)
constexpr int kScanBlock = 1024;  // elements per block of the prefix sums
constexpr int kGalWarps = 8;      // coarse rows per block of the Galerkin walk

struct Ell {
  const int* __restrict__ sp;       // slice offsets
  const uint8_t* __restrict__ sw;   // slots per slice
  const int* __restrict__ col;      // -1 = padding
};

// ---- exclusive prefix sums of int arrays -----------------------------------------
// out[k] = in[0] + ... + in[k-1] for k < n; block sums in bs.
__global__ void __launch_bounds__(kScanBlock) k_scan_block(int n, const int* __restrict__ in,
                                                           int* __restrict__ out,
                                                           int* __restrict__ bs) {
  __shared__ int wsum[kScanBlock / 32];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const long long g = (long long)blockIdx.x * kScanBlock + t;
  const int v = g < n ? in[g] : 0;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    int s = wsum[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    wsum[lane] = s;  // inclusive
  }
  __syncthreads();
  const int before = w > 0 ? wsum[w - 1] : 0;
  if (g < n) out[g] = before + x - v;
  if (t == kScanBlock - 1) bs[blockIdx.x] = before + x;
}

// Exclusive prefix sum of the nb block sums in place (one block); the total
// goes to *total.
__global__ void __launch_bounds__(kScanBlock) k_scan_sums(int nb, int* __restrict__ bs,
                                                          int* __restrict__ total) {
  __shared__ int wsum[kScanBlock / 32];
  __shared__ int carry;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  if (t == 0) carry = 0;
  __syncthreads();
  for (int c0 = 0; c0 < nb; c0 += kScanBlock) {
    const int g = c0 + t;
    const int v = g < nb ? bs[g] : 0;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
      int s = wsum[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
      }
      wsum[lane] = s;
    }
    __syncthreads();
    const int before = (w > 0 ? wsum[w - 1] : 0) + carry;
    if (g < nb) bs[g] = before + x - v;
    __syncthreads();
    if (t == kScanBlock - 1) carry = before + x;
    __syncthreads();
  }
  if (t == 0) *total = carry;
}

__global__ void k_scan_add(int n, int* __restrict__ out, const int* __restrict__ bs,
                           const int* __restrict__ total) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g < n) out[g] += bs[g / kScanBlock];
  if (g == 0) out[n] = *total;
}

// ---- handshake matching --------------------------------------------------------------
// mate[i]: -1 free, else the partner.  prop[i]: the free neighbour i proposes to.
__global__ void k_hs_propose(int n, Ell g, const float* __restrict__ w,
                             const int* __restrict__ mate, int* __restrict__ prop) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (mate[i] >= 0) {
      prop[i] = -1;
      continue;
    }
    const int s = i >> 5, base = g.sp[s] + (i & 31), ws = g.sw[s];
    int best = -1;
    float bw = 0.0f;
    for (int k = 0; k < ws; ++k) {
      const int e = base + k * 32;
      const int j = g.col[e];
      if (j < 0 || j == i || mate[j] >= 0) continue;
      const float x = w[e];
      if (x > bw || (x == bw && x > 0.0f && j < best)) {
        bw = x;
        best = j;
      }
    }
    prop[i] = best;
  }
}

__global__ void k_hs_accept(int n, const int* __restrict__ prop, int* __restrict__ mate) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int j = prop[i];
    if (mate[i] < 0 && j >= 0 && prop[j] == i) mate[i] = j;
  }
}

// rep[i]: the lower member of i's pair; a node the handshakes left alone
// stays alone, or with `join` joins the pair of its most strongly coupled
// matched neighbour (first such maximum in slot order).  flag[i] = 1 where
// i represents.
__global__ void k_hs_rep(int n, Ell g, const float* __restrict__ w, const int* __restrict__ mate,
                         int join, int* __restrict__ rep, int* __restrict__ flag) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int m = mate[i];
    int r = m >= 0 ? min(i, m) : i;
    if (m < 0 && join) {
      const int s = i >> 5, base = g.sp[s] + (i & 31), ws = g.sw[s];
      float bw = 0.0f;
      for (int k = 0; k < ws; ++k) {
        const int e = base + k * 32;
        const int j = g.col[e];
        if (j < 0 || j == i || mate[j] < 0) continue;
        if (w[e] > bw) {
          bw = w[e];
          r = min(j, mate[j]);
        }
      }
    }
    rep[i] = r;
    flag[i] = r == i ? 1 : 0;
  }
}

// agg[i] = number of i's representative
__global__ void k_hs_number(int n, const int* __restrict__ rep, const int* __restrict__ id,
                            int* __restrict__ agg) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    agg[i] = id[rep[i]];
}
__global__ void k_compose(int n, int* __restrict__ comp, const int* __restrict__ agg) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    comp[i] = agg[comp[i]];
}

// ---- aggregate sizes, singletons, members ---------------------------------------------
__global__ void k_count(int n, const int* __restrict__ agg, int* __restrict__ cnt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    atomicAdd(&cnt[agg[i]], 1);
}

// A cell alone in its aggregate joins its most strongly coupled neighbour's
// aggregate of more than one member (first such maximum in slot order).
__global__ void k_join_singletons(int n, Ell g, const float* __restrict__ w,
                                  const int* __restrict__ agg, const int* __restrict__ size,
                                  int* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int a = agg[i];
    if (size[a] == 1) {
      const int s = i >> 5, base = g.sp[s] + (i & 31), ws = g.sw[s];
      float bw = 0.0f;
      for (int k = 0; k < ws; ++k) {
        const int e = base + k * 32;
        const int j = g.col[e];
        if (j < 0 || j == i || size[agg[j]] <= 1) continue;
        if (w[e] > bw) {
          bw = w[e];
          a = agg[j];
        }
      }
    }
    out[i] = a;
  }
}

__global__ void k_mark(int n, const int* __restrict__ agg, int* __restrict__ used) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    used[agg[i]] = 1;
}
__global__ void k_renumber(int n, int* __restrict__ agg, const int* __restrict__ id) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    agg[i] = id[agg[i]];
}

// members: cells placed by an atomic cursor, then each list sorted ascending
__global__ void k_place(int n, const int* __restrict__ agg, const int* __restrict__ mptr,
                        int* __restrict__ cur, int* __restrict__ cells) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int a = agg[i];
    cells[mptr[a] + atomicAdd(&cur[a], 1)] = i;
  }
}
__global__ void k_sort_members(int nc, const int* __restrict__ mptr, int* __restrict__ cells) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nc; a += gridDim.x * blockDim.x) {
    const int b = mptr[a], e = mptr[a + 1];
    for (int p = b + 1; p < e; ++p) {
      const int x = cells[p];
      int q = p - 1;
      while (q >= b && cells[q] > x) {
        cells[q + 1] = cells[q];
        --q;
      }
      cells[q + 1] = x;
    }
  }
}

// ---- Galerkin structure ---------------------------------------------------------------
// One warp per coarse row I walks the finer slots of I's members (members
// ascending, slots ascending, 32 slots of a member at a time) and keeps the
// row's distinct neighbour aggregates in shared memory in order of first
// appearance.  MODE 0 counts them (deg), MODE 1 writes the coarse columns
// and the number of finer slots per coarse slot (cnt), MODE 2 writes the
// finer slot lists (gsrc, offsets gptr).  A row wider than kMaxRow sets
// *err.
template <int MODE>
__global__ void __launch_bounds__(kGalWarps * 32) k_galerkin(
    int nc, Ell f, const int* __restrict__ agg, const int* __restrict__ mptr,
    const int* __restrict__ cells, int* __restrict__ deg, const int* __restrict__ csp,
    int* __restrict__ ccol, int* __restrict__ cnt, const int* __restrict__ gptr,
    int* __restrict__ gsrc, int* __restrict__ err) {
  __shared__ int list[kGalWarps][kMaxRow + 1];
  __shared__ int ctr[kGalWarps][kMaxRow + 1];
  const int wi = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  for (int I = blockIdx.x * kGalWarps + wi; I < nc; I += gridDim.x * kGalWarps) {
    for (int q = lane; q <= kMaxRow; q += 32) ctr[wi][q] = 0;
    __syncwarp();
    int L = 0;
    bool over = false;
    const long long cbase = MODE > 0 ? (long long)csp[I >> 5] + (I & 31) : 0;
    for (int m = mptr[I]; m < mptr[I + 1]; ++m) {
      const int i = cells[m];
      const int s = i >> 5, ws = f.sw[s];
      const long long base = (long long)f.sp[s] + (i & 31);
      for (int k0 = 0; k0 < ws; k0 += 32) {
        const int k = k0 + lane;
        const long long e = base + (long long)k * 32;
        int J = -1;
        if (k < ws) {
          const int j = f.col[e];
          if (j >= 0) {
            J = agg[j];
            if (J == I) J = -1;
          }
        }
        int pos = -1;
        if (J >= 0)
          for (int q = 0; q < L; ++q)
            if (list[wi][q] == J) {
              pos = q;
              break;
            }
        const unsigned grp = __match_any_sync(0xffffffffu, J);
        const int leader = __ffs(grp) - 1;
        const bool fresh = J >= 0 && pos < 0 && lane == leader;
        const unsigned nb = __ballot_sync(0xffffffffu, fresh);
        if (fresh) {
          pos = L + __popc(nb & lt);
          if (pos < kMaxRow) {
            list[wi][pos] = J;
            if (MODE == 1) ccol[cbase + (long long)pos * 32] = J;
          }
        }
        const int lp = __shfl_sync(0xffffffffu, pos, leader);
        if (J >= 0 && pos < 0) pos = lp;
        L += __popc(nb);
        if (L > kMaxRow) over = true;
        if (MODE == 1 && J >= 0 && pos < kMaxRow) atomicAdd(&ctr[wi][pos], 1);
        if (MODE == 2 && J >= 0 && pos < kMaxRow) {
          const int rank = ctr[wi][pos] + __popc(grp & lt);
          gsrc[gptr[cbase + (long long)pos * 32] + rank] = (int)e;
        }
        __syncwarp();
        if (MODE == 2 && J >= 0 && pos < kMaxRow && lane == leader)
          ctr[wi][pos] += __popc(grp);
        __syncwarp();
        if (over) break;
      }
      if (over) break;
    }
    if (over) {
      if (lane == 0) atomicExch(err, 1);
      continue;
    }
    if (MODE == 0 && lane == 0) deg[I] = L;
    if (MODE == 1)
      for (int q = lane; q < L; q += 32) cnt[cbase + (long long)q * 32] = ctr[wi][q];
    __syncwarp();
  }
}

// slice widths of the coarse level: sw[s] = max deg over its 32 rows, and
// 32 sw[s] slots per slice (for the prefix sum that gives the offsets)
__global__ void k_slice_widths(int nc, const int* __restrict__ deg, uint8_t* __restrict__ sw,
                               int* __restrict__ slots) {
  const int ns = (nc + 31) / 32;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < ns; s += gridDim.x * blockDim.x) {
    int w = 0;
    for (int l = 0; l < 32; ++l)
      if (s * 32 + l < nc) w = max(w, deg[s * 32 + l]);
    sw[s] = (uint8_t)min(w, kMaxRow);
    slots[s] = 32 * w;
  }
}

// strengths of the next pass graph: |summed couplings| of the finer slots
__global__ void k_sum_abs(long long ns, const int* __restrict__ gptr, const int* __restrict__ gsrc,
                          const float* __restrict__ wf, float* __restrict__ w) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ns;
       e += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = gptr[e]; k < gptr[e + 1]; ++k) s += (double)wf[gsrc[k]];
    w[e] = (float)fabs(s);
  }
}

__global__ void k_abs(long long n, const float* __restrict__ v, float* __restrict__ w) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x)
    w[e] = fabsf(v[e]);
}

}  // namespace mgb
