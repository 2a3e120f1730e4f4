// mg.cuh -- aggregation multigrid around the learned preconditioner.
//
// A preconditioner that acts on one row at a time (the network's operator
// M^-1 = D^-1/2 S (I + E) S D^-1/2 reaches one neighbour) cannot change how
// the CG iteration count grows with the mesh: smooth error spans the whole
// domain.  Here the network's operator is the smoother on the finest level
// of an aggregation hierarchy, and one symmetric V-cycle is the
// preconditioner of flexible CG:
//
//   level l+1 cells = aggregates of about 8 level-l cells (three passes of
//                     pairwise matching along the strongest coupling),
//   P_l            = piecewise-constant prolongation (cell -> its aggregate),
//   A_{l+1}        = P^T A_l P (Galerkin: coefficients of the faces between
//                     two aggregates summed, row sums summed),
//   V-cycle on b:  x = w K b;  t = b - A x;  x += a P V(P^T t);
//                  x += w K (b - A x),
//   K              = the network's operator on level 0 (or its diagonal
//                     S^2 D^-1 alone -- learned Jacobi weights, fused like
//                     Jacobi -- or D^-1), D^-1 below,
//   coarsest level = at most kCoarsest cells, solved with its dense inverse.
//
// With a symmetric positive definite K on level 0 and Jacobi below, the
// V-cycle is a symmetric linear operator; flexible CG tolerates it being
// indefinite in rare cases, and hands over to Jacobi-PCG if a step loses
// positive curvature.
//
// Every level keeps the fine level's layout: sliced ELL rows (32 cells per
// slice, slot-major), FP32 coefficients and the FP32 row sum in place of the
// diagonal, so the product is taken in difference form
// (A x)_i = rs_i x_i + sum_j a_ij (x_j - x_i) on every level.
//
// The aggregation (structure) is computed on the host once per matrix
// structure, from the coefficients present then; the coarse coefficients
// are recomputed on the device for every solve (gathers in a fixed order,
// FP64 sums, deterministic).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <thread>
#include <vector>

#include "kernels.cuh"

namespace mg {

constexpr int kCoarsest = 256;   // dense inverse at or below this many cells
constexpr int kMaxLevels = 12;   // coarse levels at most
constexpr int kCoarseBlock = 256;

// ---- host: graphs and aggregation ---------------------------------------------
// Undirected graph in CSR with positive coupling strengths (|a_ij|).
struct Graph {
  int n = 0;
  std::vector<long long> ptr;  // n + 1
  std::vector<int> adj;
  std::vector<float> w;
};

// One pass of pairwise matching: each cell still free, in index order, is
// paired with its free neighbour of strongest coupling (ties: lowest index),
// or stays alone.  agg[i] = new index (numbered in order of creation, so
// locality of the input numbering is kept); returns the number of aggregates.
inline int match_pass(const Graph& g, std::vector<int>& agg) {
  agg.assign(g.n, -1);
  int nc = 0;
  for (int i = 0; i < g.n; ++i) {
    if (agg[i] >= 0) continue;
    int best = -1;
    float bw = 0.0f;
    for (long long k = g.ptr[i]; k < g.ptr[i + 1]; ++k) {
      const int j = g.adj[k];
      if (j == i || agg[j] >= 0) continue;
      if (g.w[k] > bw || (g.w[k] == bw && best >= 0 && j < best)) {
        bw = g.w[k];
        best = j;
      }
    }
    agg[i] = nc;
    if (best >= 0 && bw > 0.0f) agg[best] = nc;
    ++nc;
  }
  return nc;
}

// Members of each aggregate, in increasing cell index (counting sort).
inline void members(const std::vector<int>& agg, int nc, std::vector<int>& ptr,
                    std::vector<int>& cells) {
  ptr.assign(nc + 1, 0);
  for (int a : agg) ptr[a + 1]++;
  for (int k = 0; k < nc; ++k) ptr[k + 1] += ptr[k];
  cells.resize(agg.size());
  std::vector<int> pos(ptr.begin(), ptr.end() - 1);
  for (int i = 0; i < (int)agg.size(); ++i) cells[pos[agg[i]]++] = i;
}

// Run f(begin, end, thread) over [0, n) in contiguous chunks on up to 16
// host threads (one for small n).  Callers write disjoint outputs per index,
// so results do not depend on the number of threads.
template <typename F>
inline void parallel_rows(int n, F f) {
  const unsigned hc = std::thread::hardware_concurrency();
  int T = (int)std::max(1u, std::min(hc ? hc : 1u, 16u));
  if (n < 65536) T = 1;
  const int chunk = (n + T - 1) / T;
  std::vector<std::thread> th;
  for (int t = 1; t < T; ++t) {
    const int b = t * chunk, e = std::min(n, b + chunk);
    if (b < e) th.emplace_back(f, b, e, t);
  }
  f(0, std::min(n, chunk), 0);
  for (auto& x : th) x.join();
}

// Graph of the aggregates: strengths of the couplings between two
// aggregates summed (in member order, then row order), couplings inside an
// aggregate dropped; each row lists its neighbours in order of first
// appearance.
inline Graph coarsen(const Graph& g, const std::vector<int>& agg, int nc) {
  std::vector<int> mp, mc;
  members(agg, nc, mp, mc);
  Graph out;
  out.n = nc;
  out.ptr.assign(nc + 1, 0);
  const int T = 16;
  std::vector<std::vector<int>> tadj(T);
  std::vector<std::vector<float>> tw(T);
  std::vector<int> deg(nc, 0), first(T, 0);
  parallel_rows(nc, [&](int b, int e, int t) {
    std::vector<int> mark(nc, -1), pos(nc, 0);
    auto& A = tadj[t];
    auto& W = tw[t];
    first[t] = b;
    for (int I = b; I < e; ++I) {
      const size_t r0 = A.size();
      for (int m = mp[I]; m < mp[I + 1]; ++m) {
        const int i = mc[m];
        for (long long k = g.ptr[i]; k < g.ptr[i + 1]; ++k) {
          const int J = agg[g.adj[k]];
          if (J == I) continue;
          if (mark[J] != I) {
            mark[J] = I;
            pos[J] = (int)(A.size() - r0);
            A.push_back(J);
            W.push_back(g.w[k]);
          } else {
            W[r0 + pos[J]] += g.w[k];
          }
        }
      }
      deg[I] = (int)(A.size() - r0);
    }
  });
  for (int I = 0; I < nc; ++I) out.ptr[I + 1] = out.ptr[I] + deg[I];
  out.adj.resize(out.ptr[nc]);
  out.w.resize(out.ptr[nc]);
  for (int t = 0; t < T; ++t) {
    if (tadj[t].empty()) continue;
    std::copy(tadj[t].begin(), tadj[t].end(), out.adj.begin() + out.ptr[first[t]]);
    std::copy(tw[t].begin(), tw[t].end(), out.w.begin() + out.ptr[first[t]]);
  }
  return out;
}

// Aggregates of about 2^passes cells: passes of matching, composed.  A cell
// left alone by every pass (its neighbours were all taken before its turn)
// then joins the aggregate of its most strongly coupled neighbour: left
// alone, such cells carry over from level to level and, on the small
// levels, stall the coarsening.  Aggregates keep the order of their first
// member.
inline int aggregate(const Graph& g, int passes, std::vector<int>& agg) {
  agg.resize(g.n);
  std::iota(agg.begin(), agg.end(), 0);
  Graph cur;
  const Graph* gp = &g;
  int nc = g.n;
  for (int p = 0; p < passes; ++p) {
    std::vector<int> a;
    const int n2 = match_pass(*gp, a);
    for (int& x : agg) x = a[x];
    if (p + 1 < passes) {
      cur = coarsen(*gp, a, n2);
      gp = &cur;
    }
    nc = n2;
  }
  std::vector<int> size(nc, 0);
  for (int x : agg) size[x]++;
  for (int i = 0; i < g.n; ++i) {
    if (size[agg[i]] != 1) continue;
    int best = -1;
    float bw = 0.0f;
    for (long long k = g.ptr[i]; k < g.ptr[i + 1]; ++k) {
      const int j = g.adj[k];
      if (j != i && size[agg[j]] > 1 && g.w[k] > bw) {
        bw = g.w[k];
        best = j;
      }
    }
    if (best >= 0) {
      size[agg[i]] = 0;
      agg[i] = agg[best];
      size[agg[i]]++;
    }
  }
  std::vector<int> renum(nc, -1);
  int m = 0;
  for (int i = 0; i < g.n; ++i)
    if (renum[agg[i]] < 0) renum[agg[i]] = m++;
  for (int& x : agg) x = renum[x];
  return m;
}

// Sliced-ELL structure of one coarse level and, per coarse slot, the list of
// finer-level slots whose coefficients sum into it.
struct CoarseHost {
  int n = 0;
  std::vector<int> slice_ptr;
  std::vector<uint8_t> slice_w;
  std::vector<int> col;         // -1 = padding
  std::vector<int> gptr, gsrc;  // slot e sums finer slots gsrc[gptr[e] .. gptr[e+1])
  std::vector<int> agg_ptr, agg_cells, agg_of;
  long long n_slots = 0;
};

// Fine level given by its sliced-ELL arrays (n cells) and aggregation agg.
// Coarse row I lists its neighbours J in order of first appearance over
// I's members and their slots; slot (I, J) sums the finer slots listed for
// it, in the same order.
inline bool build_coarse(int n, const std::vector<int>& sp, const std::vector<uint8_t>& sw,
                         const std::vector<int>& col, const std::vector<int>& agg, int nc,
                         CoarseHost& C) {
  C.n = nc;
  C.agg_of = agg;
  members(agg, nc, C.agg_ptr, C.agg_cells);
  const std::vector<int>& mp = C.agg_ptr;
  const std::vector<int>& mc = C.agg_cells;
  // walk the finer slots of coarse row I: visit(J, finer slot, k of J)
  auto walk = [&](int I, std::vector<int>& mark, std::vector<int>& pos, auto&& visit) {
    int d = 0;
    for (int m = mp[I]; m < mp[I + 1]; ++m) {
      const int i = mc[m];
      const int s = i >> 5, l = i & 31;
      for (int k = 0; k < sw[s]; ++k) {
        const long long e = (long long)sp[s] + (long long)k * 32 + l;
        const int j = col[e];
        if (j < 0) continue;
        const int J = agg[j];
        if (J == I) continue;
        if (mark[J] != I) {
          mark[J] = I;
          pos[J] = d++;
        }
        visit(J, (int)e, pos[J]);
      }
    }
    return d;
  };
  std::vector<int> deg(nc, 0);
  parallel_rows(nc, [&](int b, int e, int) {
    std::vector<int> mark(nc, -1), pos(nc, 0);
    for (int I = b; I < e; ++I) deg[I] = walk(I, mark, pos, [](int, int, int) {});
  });
  const int ns = (nc + 31) / 32;
  C.slice_ptr.assign(ns + 1, 0);
  C.slice_w.assign(ns, 0);
  long long total = 0;
  for (int s = 0; s < ns; ++s) {
    int w = 0;
    for (int l = 0; l < 32; ++l)
      if (s * 32 + l < nc) w = std::max(w, deg[s * 32 + l]);
    if (w > 255) return false;
    C.slice_w[s] = (uint8_t)w;
    C.slice_ptr[s] = (int)total;
    total += 32LL * w;
    if (total > (1LL << 31) - 1) return false;
  }
  C.slice_ptr[ns] = (int)total;
  C.n_slots = total;
  C.col.assign(total, -1);
  std::vector<int> cnt(total, 0);
  parallel_rows(nc, [&](int b, int e, int) {
    std::vector<int> mark(nc, -1), pos(nc, 0);
    for (int I = b; I < e; ++I) {
      const long long base = (long long)C.slice_ptr[I >> 5] + (I & 31);
      walk(I, mark, pos, [&](int J, int, int k) {
        C.col[base + (long long)k * 32] = J;
        cnt[base + (long long)k * 32]++;
      });
    }
  });
  C.gptr.assign(total + 1, 0);
  for (long long e = 0; e < total; ++e) C.gptr[e + 1] = C.gptr[e] + cnt[e];
  C.gsrc.assign(C.gptr[total], 0);
  parallel_rows(nc, [&](int b, int e, int) {
    std::vector<int> mark(nc, -1), pos(nc, 0);
    for (int I = b; I < e; ++I) {
      const long long base = (long long)C.slice_ptr[I >> 5] + (I & 31);
      std::vector<int> fill;
      walk(I, mark, pos, [&](int, int ef, int k) {
        if ((int)fill.size() <= k) fill.resize(k + 1, 0);
        const long long ec = base + (long long)k * 32;
        C.gsrc[C.gptr[ec] + fill[k]++] = ef;
      });
    }
  });
  (void)n;
  return true;
}

// Coupling graph of a level given by its sliced-ELL arrays and coefficients.
inline Graph graph_of(int n, const std::vector<int>& sp, const std::vector<uint8_t>& sw,
                      const std::vector<int>& col, const std::vector<float>& val) {
  Graph g;
  g.n = n;
  g.ptr.assign(n + 1, 0);
  std::vector<int> deg(n, 0);
  parallel_rows(n, [&](int b, int e, int) {
    for (int i = b; i < e; ++i) {
      const int s = i >> 5, l = i & 31;
      int d = 0;
      for (int k = 0; k < sw[s]; ++k) d += col[(long long)sp[s] + (long long)k * 32 + l] >= 0;
      deg[i] = d;
    }
  });
  for (int i = 0; i < n; ++i) g.ptr[i + 1] = g.ptr[i] + deg[i];
  g.adj.resize(g.ptr[n]);
  g.w.resize(g.ptr[n]);
  parallel_rows(n, [&](int b, int e, int) {
    for (int i = b; i < e; ++i) {
      const int s = i >> 5, l = i & 31;
      long long o = g.ptr[i];
      for (int k = 0; k < sw[s]; ++k) {
        const long long q = (long long)sp[s] + (long long)k * 32 + l;
        if (col[q] >= 0) {
          g.adj[o] = col[q];
          g.w[o++] = std::fabs(val[q]);
        }
      }
    }
  });
  return g;
}

// ---- device: coefficients of the coarse levels ---------------------------------
// v[e] = sum of the finer coefficients listed for slot e (FP64 sum, in list order).
__global__ void k_mg_gather_slots(long long ns, const int* __restrict__ gptr,
                                  const int* __restrict__ gsrc, const float* __restrict__ vf,
                                  float* __restrict__ v) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ns;
       e += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = gptr[e]; k < gptr[e + 1]; ++k) s += (double)vf[gsrc[k]];
    v[e] = (float)s;
  }
}

// rs[I] = sum of the finer row sums of I's members (the Galerkin row sum).
__global__ void k_mg_rowsum(int nc, const int* __restrict__ aptr, const int* __restrict__ acell,
                            const float* __restrict__ rsf, float* __restrict__ rs) {
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nc; I += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int m = aptr[I]; m < aptr[I + 1]; ++m) s += (double)rsf[acell[m]];
    rs[I] = (float)s;
  }
}

// dinv = 1 / (rs - sum_j a_ij): the inverse diagonal (0 where it is not > 0).
__global__ void k_mg_dinv(int n, sg::Rows<float> R, float* __restrict__ dinv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    sg::RowIt<float> it(R, i);
    double d = R.diag[i];
    for (int k = 0; k < it.w; ++k) {
      const int e = it.base + k * sg::kWarp;
      if (R.col[e] >= 0) d -= (double)R.val[e];
    }
    dinv[i] = d > 0.0 ? (float)(1.0 / d) : 0.0f;
  }
}

// Dense FP64 copy of the coarsest matrix (row-major n x n).
__global__ void k_mg_dense(int n, sg::Rows<float> R, double* __restrict__ A) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    for (int j = 0; j < n; ++j) A[(size_t)i * n + j] = 0.0;
    sg::RowIt<float> it(R, i);
    double d = R.diag[i];
    for (int k = 0; k < it.w; ++k) {
      const int e = it.base + k * sg::kWarp;
      const int j = R.col[e];
      if (j >= 0) {
        A[(size_t)i * n + j] += (double)R.val[e];
        d -= (double)R.val[e];
      }
    }
    A[(size_t)i * n + i] += d;
  }
}

// In-place Gauss-Jordan inverse of the symmetric positive definite coarsest
// matrix (no pivoting needed), one block; a pivot below 1e-13 of the largest
// diagonal (a singular, all-Neumann system) drops that row and column,
// which leaves a generalised inverse.  Result rounded to FP32.
__global__ void __launch_bounds__(1024)
k_mg_invert(int n, double* __restrict__ A, float* __restrict__ Ainv) {
  __shared__ double f[kCoarsest];
  __shared__ double dmax;
  __shared__ bool skip;
  const int t = threadIdx.x, nt = blockDim.x;
  if (t == 0) {
    double m = 0.0;
    for (int i = 0; i < n; ++i) m = fmax(m, fabs(A[(size_t)i * n + i]));
    dmax = m;
  }
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    if (t == 0) skip = !(fabs(A[(size_t)k * n + k]) > 1e-13 * dmax);
    __syncthreads();
    if (skip) {
      for (int j = t; j < n; j += nt) {
        A[(size_t)k * n + j] = 0.0;
        A[(size_t)j * n + k] = 0.0;
      }
      __syncthreads();
      continue;
    }
    const double ip = 1.0 / A[(size_t)k * n + k];
    __syncthreads();
    for (int j = t; j < n; j += nt) A[(size_t)k * n + j] = (j == k) ? ip : A[(size_t)k * n + j] * ip;
    for (int i = t; i < n; i += nt) f[i] = (i == k) ? 0.0 : A[(size_t)i * n + k];
    __syncthreads();
    for (int q = t; q < n * n; q += nt) {
      const int i = q / n, j = q % n;
      if (i == k) continue;
      const double a = (j == k) ? 0.0 : A[q];
      A[q] = a - f[i] * A[(size_t)k * n + j];
    }
    __syncthreads();
  }
  for (int q = t; q < n * n; q += nt) Ainv[q] = (float)A[q];
}

// ---- device: the V-cycle ---------------------------------------------------------
// x = w D^-1 b and t = b - A x (pre-smoothing from zero, then its residual;
// x_j at the neighbours is recomputed from b_j).
template <int CH = sg::kRowChunk>
__global__ void k_mg_pre(int n, sg::Rows<float> R, const float* __restrict__ dinv, float w,
                         const float* __restrict__ b, float* __restrict__ x,
                         float* __restrict__ t, const int* __restrict__ n_active) {
  if (n_active && *n_active == 0) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    sg::RowIt<float> it(R, i);
    const float bi = b[i];
    const float xi = w * dinv[i] * bi;
    float y = R.diag[i] * xi;
    for (int k0 = 0; k0 < it.w; k0 += CH) {
      int j[CH];
      float a[CH], xj[CH];
#pragma unroll
      for (int u = 0; u < CH; ++u) {
        j[u] = -1;
        a[u] = 0.0f;
        if (k0 + u < it.w) {
          const int e = it.base + (k0 + u) * sg::kWarp;
          j[u] = __ldg(&R.col[e]);
          a[u] = R.val[e];
        }
      }
#pragma unroll
      for (int u = 0; u < CH; ++u) xj[u] = j[u] >= 0 ? w * dinv[j[u]] * b[j[u]] : xi;
#pragma unroll
      for (int u = 0; u < CH; ++u)
        if (j[u] >= 0) y = fmaf(a[u], xj[u] - xi, y);
    }
    x[i] = xi;
    t[i] = bi - y;
  }
}

// t = b - A x
template <int CH = sg::kRowChunk>
__global__ void k_mg_resid(int n, sg::Rows<float> R, const float* __restrict__ b,
                           const float* __restrict__ x, float* __restrict__ t,
                           const int* __restrict__ n_active) {
  if (n_active && *n_active == 0) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float y[1];
    sg::row_apply<float, 1, CH>(R, i, x, y);
    t[i] = b[i] - y[0];
  }
}

// y = x + w D^-1 (b - A x)  (post-smoothing; y and x are different arrays)
template <typename TO, int CH = sg::kRowChunk>
__global__ void k_mg_post(int n, sg::Rows<float> R, const float* __restrict__ dinv, float w,
                          const float* __restrict__ b, const float* __restrict__ x,
                          TO* __restrict__ y, const int* __restrict__ n_active) {
  if (n_active && *n_active == 0) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float ax[1];
    sg::row_apply<float, 1, CH>(R, i, x, ax);
    y[i] = (TO)(x[i] + w * dinv[i] * (b[i] - ax[0]));
  }
}

// The network's operator as smoother: out = [out +] w K in,
// K in = q (q in + E (q in)) (the learned preconditioner's application).
template <bool ADD, typename TO>
__global__ void k_mg_net(int n, sg::Rows<float> R, const float* __restrict__ gE,
                         const float* __restrict__ q, float w, const float* __restrict__ in,
                         const float* __restrict__ base, TO* __restrict__ out,
                         const int* __restrict__ n_active) {
  if (n_active && *n_active == 0) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    sg::RowIt<float> it(R, i);
    const float qi = q[i];
    float t = qi * in[i];
    for (int k0 = 0; k0 < it.w; k0 += sg::kRowChunk) {
      int j[sg::kRowChunk];
      float g[sg::kRowChunk], qj[sg::kRowChunk], vj[sg::kRowChunk];
#pragma unroll
      for (int u = 0; u < sg::kRowChunk; ++u) {
        j[u] = -1;
        g[u] = 0.0f;
        if (k0 + u < it.w) {
          const int e = it.base + (k0 + u) * sg::kWarp;
          j[u] = __ldg(&R.col[e]);
          g[u] = gE[e];
        }
      }
#pragma unroll
      for (int u = 0; u < sg::kRowChunk; ++u) {
        qj[u] = j[u] >= 0 ? q[j[u]] : 0.0f;
        vj[u] = j[u] >= 0 ? in[j[u]] : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < sg::kRowChunk; ++u)
        if (j[u] >= 0) t = fmaf(g[u] * qj[u], vj[u], t);
    }
    const float v = w * qi * t;
    out[i] = (TO)(ADD ? base[i] + v : v);
  }
}

// ---- device: bounding the network smoother -----------------------------------------
// v_i = a fixed pseudo-random value in [-1, 1) (power-iteration start)
__global__ void k_mg_hashfill(int n, float* __restrict__ v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    unsigned int h = (unsigned int)i * 2654435761u + 0x9e3779b9u;
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    v[i] = (float)(h & 0xFFFFFF) * (2.0f / 16777216.0f) - 1.0f;
  }
}

// out += x.x (FP64, one atomic per block)
__global__ void __launch_bounds__(256) k_mg_norm2(int n, const float* __restrict__ x,
                                                  double* __restrict__ out) {
  __shared__ double sh[8];
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    acc += (double)x[i] * x[i];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sh[k];
    atomicAdd(out, t);
  }
}

// q_i = max(q_i, f rsd_i): the network's per-cell scale s = q / rsd held at
// or above f, so no cell is left (almost) unsmoothed.  A NaN stays NaN: a
// broken network must reach flexible CG's hand-over to plain PCG, not be
// quietly repaired here.
__global__ void k_mg_floor(int n, float f, const float* __restrict__ rsd, float* __restrict__ q) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float lo = f * rsd[i];
    if (q[i] < lo) q[i] = lo;
  }
}

// x *= c
__global__ void k_mg_scale(int n, float c, float* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] *= c;
}

// dq = q^2: the network's per-cell scale as a Jacobi weight (smoother 2)
__global__ void k_mg_square(int n, const float* __restrict__ q, float* __restrict__ dq) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    dq[i] = q[i] * q[i];
}

// bc[I] = sum of t over I's members (restriction P^T)
__global__ void k_mg_restrict(int nc, const int* __restrict__ aptr,
                              const int* __restrict__ acell, const float* __restrict__ t,
                              float* __restrict__ bc, const int* __restrict__ n_active) {
  if (n_active && *n_active == 0) return;
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < nc; I += gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int m = aptr[I]; m < aptr[I + 1]; ++m) s += t[acell[m]];
    bc[I] = s;
  }
}

// x[i] += a xc[agg_of[i]]  (prolongation P, scaled)
__global__ void k_mg_prolong(int n, const int* __restrict__ agg_of, float a,
                             const float* __restrict__ xc, float* __restrict__ x,
                             const int* __restrict__ n_active) {
  if (n_active && *n_active == 0) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] += a * xc[agg_of[i]];
}

// x = Ainv b on the coarsest level (one block)
__global__ void __launch_bounds__(kCoarseBlock)
k_mg_coarse_solve(int n, const float* __restrict__ Ainv, const float* __restrict__ b,
                  float* __restrict__ x, const int* __restrict__ n_active) {
  if (n_active && *n_active == 0) return;
  __shared__ float sb[kCoarsest];
  for (int j = threadIdx.x; j < n; j += blockDim.x) sb[j] = b[j];
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    float s = 0.0f;
    for (int j = 0; j < n; ++j) s = fmaf(Ainv[(size_t)i * n + j], sb[j], s);
    x[i] = s;
  }
}

// ---- device: training the network through the V-cycle ----------------------------
// Loss per sample b (original space, z = V(b)): L = -log((z.b)^2 / (z.A z)).
// (z.b)^2/(z.Az) is twice the energy one CG step along z removes -- free of
// z's overall scale; the logarithm makes every sample count alike whatever
// its own energy, which varies by orders of magnitude between smooth and
// rough residuals.

// b = r / gs (the sample at unit mean scaled magnitude; gs in lane 0)
__global__ void k_mg_normalise(int n, const float* __restrict__ r, const sg::Lane* __restrict__ lanes,
                               float* __restrict__ b) {
  const double gs = lanes[0].gs > 0 ? lanes[0].gs : 1.0;
  const float inv = (float)(1.0 / gs);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    b[i] = r[i] * inv;
}

// az = A z; sums[0] += z.b, sums[1] += z.az (FP64; one atomic per block)
__global__ void __launch_bounds__(256)
k_mg_loss_sums(int n, sg::Rows<float> R, const float* __restrict__ z, const float* __restrict__ b,
               float* __restrict__ az, double* __restrict__ sums) {
  __shared__ double sh[2][8];
  double zb = 0.0, zaz = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float y[1];
    sg::row_apply<float, 1>(R, i, z, y);
    az[i] = y[0];
    zb += (double)z[i] * b[i];
    zaz += (double)z[i] * y[0];
  }
  for (int o = 16; o > 0; o >>= 1) {
    zb += __shfl_down_sync(0xffffffffu, zb, o);
    zaz += __shfl_down_sync(0xffffffffu, zaz, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { sh[0][w] = zb; sh[1][w] = zaz; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, c = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { a += sh[0][k]; c += sh[1][k]; }
    atomicAdd(&sums[0], a);
    atomicAdd(&sums[1], c);
  }
}

// g = dL/dz = 2 (A z / (z.Az) - b / (z.b)); jsum += L (once)
__global__ void k_mg_loss_grad(int n, const float* __restrict__ az, const float* __restrict__ b,
                               const double* __restrict__ sums, float* __restrict__ g,
                               double* __restrict__ jsum) {
  const double zb = sums[0], zaz = sums[1];
  // a sample whose z is (numerically) orthogonal to b or not finite has no
  // usable gradient (2/z.b explodes): it is skipped
  const bool ok = zaz > 0.0 && isfinite(zaz) && isfinite(zb) && zb * zb > 1e-20 * zaz;
  const float ca = ok ? (float)(2.0 / zaz) : 0.0f, cb = ok ? (float)(2.0 / zb) : 0.0f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    g[i] = ca * az[i] - cb * b[i];
  if (blockIdx.x == 0 && threadIdx.x == 0 && ok) *jsum += -log(zb * zb / zaz);
}

// One application x -> w K x of the smoother, K = D^-1/2 S (I+E) S D^-1/2,
// seen from the scaled-space backward kernels: input u = rsd x and output
// gradient gh = w rsd g (g the gradient with respect to w K x).
__global__ void k_mg_scaled_pair(int n, const float* __restrict__ rsd, float w,
                                 const float* __restrict__ x, const float* __restrict__ g,
                                 float* __restrict__ u, float* __restrict__ gh) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    u[i] = rsd[i] * x[i];
    gh[i] = w * rsd[i] * g[i];
  }
}

}  // namespace mg
