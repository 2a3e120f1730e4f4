// solv_gpu.cu -- host runtime and C-ABI of the B200 face-addressed Krylov
// solvers (include/solv_gpu.h).
//
// Hot path replaced: spray-simulation/solv_cg.f90, solv_bicg.f90,
// solv_precond.f90, solv_direct.f90, solv_res.f90 over the matrix of
// solv_data.f90 (ng, pl, v_lst).  The matrix is copied to HBM once per
// structure, re-laid out (wavefront-level-major cell order, sliced ELL
// rows in face order) and kept resident; solves run as a chain of fused
// kernels with the Krylov scalars kept on the device, so the host only
// polls a convergence counter every `graph_iters` iterations.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include "../../include/solv_gpu.h"
#include "kernels.cuh"
#include "gnn.cuh"
#include "mg.cuh"
#include "mg_build.cuh"

using sg::Lane;
using sg::Rows;
using sg::SegMap;

namespace {

constexpr int kMaxV = 4;

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { if (p) cudaFree(p); }
  void swap(DevBuf& o) {
    std::swap(p, o.p);
    std::swap(bytes, o.bytes);
  }
  void release() { if (p) cudaFree(p); p = nullptr; bytes = 0; }
  cudaError_t ensure(size_t b) {
    if (b <= bytes && p) return cudaSuccess;
    release();
    cudaError_t e = cudaMalloc(&p, b ? b : 16);
    if (e == cudaSuccess) bytes = b;
    return e;
  }
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

// One coarse level of the aggregation hierarchy (mg.cuh); level l's
// aggregation arrays map level l-1 cells to level l cells.
struct MgLevel {
  int n = 0;
  long long n_slots = 0;
  DevBuf slice_ptr, slice_w, col, val, rs, dinv;
  DevBuf gptr, gsrc;                  // coarse slot <- finer slots
  DevBuf agg_ptr, agg_cells, agg_of;  // members (finer numbering); finer cell -> cell
  DevBuf x, b, t, y;                  // V-cycle vectors
  Rows<float> rows() const {
    Rows<float> R;
    R.slice_ptr = slice_ptr.as<int>();
    R.slice_w = slice_w.as<uint8_t>();
    R.col = col.as<int>();
    R.val = val.as<float>();
    R.sval = val.as<float>();
    R.diag = rs.as<float>();
    return R;
  }
};

// Host-side description of the segment (system) -> block map.
struct SegHost {
  std::vector<int> blk_seg, blk_rank, seg_nblk, seg_blk0, seg_c0, seg_c1;
  int total_blk = 0;
};

}  // namespace

struct solv_gpu_ctx {
  int dev = 0;
  cudaStream_t own = nullptr;
  cudaStream_t stream = nullptr;
  std::string err;
  int n_sm = 148;
  // options
  int precision = 0;
  double inner_reduc = 1e-6;
  int graph_iters = 16;
  int block = 256;
  int grid_per_sm = 8;
  int max_refine = 30;
  int inner_max_iter = 2000;
  double reliable_delta = 0.1;
  double fcg_reliable_delta = 0.1;  // the learned flexible CG's reliable-update drop
  int fcg_fallback_imat = 0;         // the PCG a stalled learned solve hands over to
  int fcg_slow_iters = 15;           // network smoother -> Jacobi after this many
                                     // iterations for one reliable-update drop (0: never)
  int smoother_switches = 0;         // of the last learned solve
  int gnn_loss = 1;  // training loss: 0 energy, 1 scale-free (best-step energy)

  // matrix (caller sizes)
  bool has_matrix = false;
  int N = 0, F = 0;
  bool orient_std = true;
  int n_seg = 1;             // independent systems (block-diagonal batch)
  std::vector<int> lvl_ptr;  // cells per wavefront level (counts, for the statistics)
  std::vector<int> seg_c0_caller, seg_c1_caller;  // system ranges in internal order
  long long n_slots = 0;
  int n_slice = 0;
  DevBuf old_of_new, slice_ptr, slice_w, col, slot_src, val, sval, diag, fp, fn;
  DevBuf valf, svalf, diagf;  // FP32 copies for the mixed-precision inner solve
  bool f32_valid = false;

  // segment map (single system: one segment)
  SegHost seg;
  DevBuf d_seg;  // packed ints
  DevBuf ticket, n_active, lanes, part, l1, mp_mask;
  int* h_n_active = nullptr;  // pinned

  // workspace
  DevBuf w_phi, w_r0, w_r, w_p, w_q, w_v, w_z, w_c, w_cr, w_in, w_out;
  DevBuf wf_r, wf_p, wf_q, wf_v, wf_z, wf_phi, wf_c, wf_cr, wf_r0;  // FP32
  DevBuf w_x, w_b;  // solv_gpu_direct / spmv staging
  // triangular sweeps (kernels.cuh, sync-free recurrences): the forward
  // sweep's output t, all "pending" between sweeps; the wait-timeout flag
  DevBuf w_t, wf_t;
  bool t_ready = false, tf_ready = false;  // t / tf hold only the pending pattern
  DevBuf sweep_ctl;
  std::map<const void*, int> coop_blocks;  // resident blocks per SM, per sweep kernel

  // captured iteration graphs, keyed by (solver, imat, V, fp32)
  std::map<std::tuple<int, int, int, int, int>, cudaGraphExec_t> graphs;  // last: 1 = WHILE graph
  bool cond_graphs = true;             // conditional WHILE graphs usable here
  int graph_loop = 2;                  // SOLV_OPT_GRAPH_LOOP: 1 WHILE graphs, 0 K per launch,
                                       // 2 WHILE for the learned FCG only
  DevBuf loop_budget;                  // iterations left in the running WHILE graph
  int launches = 0;

  cudaEvent_t ev0 = nullptr, ev1 = nullptr;

  // learned preconditioner (gnn.cuh)
  DevBuf g_param, g_grad, g_m, g_v, g_wcat;  // FP32 master, grads, Adam moments, BF16 packed
  DevBuf g_rsd, g_frs, g_fdeg, g_gw;         // per-matrix features
  DevBuf g_h0, g_h1, g_u, g_r, g_out, g_jsum, g_q, g_he, g_ge;
  DevBuf g_train;                            // training activations
  bool g_feat_valid = false, g_wcat_valid = false, g_has_params = false;
  int g_adam_t = 0;
  int fallbacks = 0;

  // aggregation multigrid around the learned preconditioner (mg.cuh)
  int mg_max_levels = mg::kMaxLevels;  // coarse levels at most; 0 = one-level preconditioner
  int mg_smoother = 1;                 // level-0 smoother: 1 the network's operator K,
                                       // 2 its diagonal (learned Jacobi weights), 0 Jacobi
  double mg_omega = 0.8;               // smoother damping (1.0 loses the V-cycle)
  double mg_alpha = 2.0;               // coarse-correction scale (unsmoothed
                                       // aggregation under-corrects smooth error)
  int mg_build = 0;                    // hierarchy build: 0 on the GPU, 1 on the host
  bool mg_valid = false;               // hierarchy built for the current structure
  int mg_built_max = 0;                // mg_max_levels the hierarchy was built with
  std::vector<std::unique_ptr<MgLevel>> mg;  // coarse levels 1..L
  DevBuf mg_x0, mg_t0, mg_dinv0, mg_dense, mg_ainv;
  DevBuf mg_train;                     // training through the V-cycle: 8 vectors
  DevBuf mg_dq;                        // smoother 2: the network's per-cell weights q^2
  DevBuf g_zero;                       // smoother 2 training: face weights held at zero
  double mg_setup_s = 0.0;
  double mg_smooth_scale = 1.0;        // factor the last solve applied to K (see mg_bound_smoother)
  float mg_scale_min = 0.5f;           // floor on the network's per-cell scales
  // the learned preconditioner hands over to Jacobi-PCG when its residual
  // stalls: fcg_stall_iters iterations without falling below fcg_stall_drop
  // times the value at the start of the window
  int row_chunk = sg::kRowChunk;       // FP32 products: matrix slots a thread loads per step
  int persistent = 0;                  // FP64 Jacobi PCG as one cluster-persistent launch
  std::map<const void*, int> pcg_max16;  // clusters of 16 resident at once, per kernel
  std::map<int, double> pcg_local;       // share of slots within their own block of 2^k cells
  int gnn_layer_blocks = 0;              // resident blocks per SM of k_gnn_layer_tc
  int fcg_stall_iters = 1000;
  double fcg_stall_drop = 0.9;
};

namespace {

int set_err(solv_gpu_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

#define CUDA_TRY(ctx, expr)                                                   \
  do {                                                                        \
    cudaError_t e_ = (expr);                                                  \
    if (e_ != cudaSuccess)                                                    \
      return set_err(ctx, SOLV_GPU_DEVICE_ERROR,                              \
                     std::string(#expr) + ": " + cudaGetErrorString(e_));     \
  } while (0)

void drop_graphs(solv_gpu_ctx* c) {
  for (auto& kv : c->graphs)
    if (kv.second) cudaGraphExecDestroy(kv.second);
  c->graphs.clear();
}

SegMap segmap(solv_gpu_ctx* c) {
  const int nb = c->seg.total_blk, ns = (int)c->seg.seg_nblk.size();
  int* base = c->d_seg.as<int>();
  SegMap m;
  m.blk_seg = base;
  m.blk_rank = base + nb;
  m.seg_nblk = base + 2 * nb;
  m.seg_blk0 = base + 2 * nb + ns;
  m.seg_c0 = base + 2 * nb + 2 * ns;
  m.seg_c1 = base + 2 * nb + 3 * ns;
  m.ticket = c->ticket.as<unsigned int>();
  m.n_active = c->n_active.as<int>();
  return m;
}

// Blocks per segment proportional to its size, at least one each.
int build_segments(solv_gpu_ctx* c, const std::vector<int>& seg_c0,
                   const std::vector<int>& seg_c1) {
  SegHost& s = c->seg;
  s = SegHost();
  const int ns = (int)seg_c0.size();
  long long total = 0;
  for (int k = 0; k < ns; ++k) total += seg_c1[k] - seg_c0[k];
  // all blocks of the reduction grid resident: at most 2048 threads per SM
  const long long per_sm = std::min(c->grid_per_sm, 2048 / c->block);
  const long long cap = (long long)c->n_sm * std::max(1LL, per_sm);
  for (int k = 0; k < ns; ++k) {
    long long n = seg_c1[k] - seg_c0[k];
    long long want = (n + c->block - 1) / c->block;
    long long share = total > 0 ? (cap * n + total - 1) / total : 1;
    int nb = (int)std::max(1LL, std::min(want, share));
    s.seg_blk0.push_back(s.total_blk);
    s.seg_nblk.push_back(nb);
    s.seg_c0.push_back(seg_c0[k]);
    s.seg_c1.push_back(seg_c1[k]);
    for (int r = 0; r < nb; ++r) {
      s.blk_seg.push_back(k);
      s.blk_rank.push_back(r);
    }
    s.total_blk += nb;
  }
  std::vector<int> packed;
  packed.insert(packed.end(), s.blk_seg.begin(), s.blk_seg.end());
  packed.insert(packed.end(), s.blk_rank.begin(), s.blk_rank.end());
  packed.insert(packed.end(), s.seg_nblk.begin(), s.seg_nblk.end());
  packed.insert(packed.end(), s.seg_blk0.begin(), s.seg_blk0.end());
  packed.insert(packed.end(), s.seg_c0.begin(), s.seg_c0.end());
  packed.insert(packed.end(), s.seg_c1.begin(), s.seg_c1.end());
  CUDA_TRY(c, c->d_seg.ensure(packed.size() * sizeof(int)));
  CUDA_TRY(c, cudaMemcpyAsync(c->d_seg.p, packed.data(), packed.size() * sizeof(int),
                              cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, c->ticket.ensure(ns * sizeof(unsigned)));
  CUDA_TRY(c, cudaMemsetAsync(c->ticket.p, 0, ns * sizeof(unsigned), c->stream));
  CUDA_TRY(c, c->lanes.ensure((size_t)ns * kMaxV * sizeof(Lane)));
  CUDA_TRY(c, c->l1.ensure((size_t)ns * kMaxV * sizeof(double)));
  CUDA_TRY(c, c->part.ensure((size_t)s.total_blk * 2 * kMaxV * sizeof(double)));
  CUDA_TRY(c, c->n_active.ensure(sizeof(int)));
  drop_graphs(c);
  return SOLV_GPU_OK;
}

template <typename T>
Rows<T> rows(solv_gpu_ctx* c) {
  Rows<T> R;
  R.slice_ptr = c->slice_ptr.as<int>();
  R.slice_w = c->slice_w.as<uint8_t>();
  R.col = c->col.as<int>();
  if constexpr (std::is_same<T, double>::value) {
    R.val = c->val.as<double>();
    R.sval = c->orient_std ? c->val.as<double>() : c->sval.as<double>();
    R.diag = c->diag.as<double>();
  } else {
    R.val = c->valf.as<float>();
    R.sval = c->orient_std ? c->valf.as<float>() : c->svalf.as<float>();
    R.diag = c->diagf.as<float>();
  }
  return R;
}

int grid_for(solv_gpu_ctx* c, long long n) {
  long long g = (n + c->block - 1) / c->block;
  long long cap = (long long)c->n_sm * 16;
  return (int)std::max(1LL, std::min(g, cap));
}

// Grid of the grid-stride matrix products: one full wave (2048 threads per
// SM), so no block is left for a second, nearly empty wave.
int grid_resident(solv_gpu_ctx* c, long long n) {
  long long g = (n + c->block - 1) / c->block;
  long long cap = (long long)c->n_sm * std::max(1, 2048 / c->block);
  return (int)std::max(1LL, std::min(g, cap));
}


// Run f with the FP32 products' gather width (slots loaded per step) as a
// compile-time constant: f(std::integral_constant<int, CH>()).
template <typename F>
void with_chunk(int ch, F&& f) {
  switch (ch) {
    case 2: f(std::integral_constant<int, 2>()); break;
    case 8: f(std::integral_constant<int, 8>()); break;
    default: f(std::integral_constant<int, 4>()); break;
  }
}

// ---- matrix structure --------------------------------------------------------
int matrix_structure(solv_gpu_ctx* c, int N, int F, const int* ip, const int* in, int nsys,
                     const int* cell_ptr) {
  if (N <= 0 || F < 0 || !ip || !in || nsys < 1)
    return set_err(c, SOLV_GPU_BAD_INPUT, "matrix_set: bad sizes or null pointers");
  std::vector<int> seg_of(N, 0);
  if (nsys > 1) {
    if (!cell_ptr || cell_ptr[0] != 0 || cell_ptr[nsys] != N)
      return set_err(c, SOLV_GPU_BAD_INPUT, "matrix_set_batch: cell_ptr must run 0..n_cell");
    for (int k = 0; k < nsys; ++k) {
      if (cell_ptr[k + 1] <= cell_ptr[k])
        return set_err(c, SOLV_GPU_BAD_INPUT, "matrix_set_batch: empty or unordered system");
      for (int i = cell_ptr[k]; i < cell_ptr[k + 1]; ++i) seg_of[i] = k;
    }
  }
  // validate + per-cell interior degree
  std::vector<int> deg(N, 0);
  bool orient = true;
  for (int f = 0; f < F; ++f) {
    int a = ip[f], b = in[f];
    if (a < 1 || a > N || b < 0 || b > N || a == b)
      return set_err(c, SOLV_GPU_BAD_INPUT,
                     "matrix_set: face " + std::to_string(f + 1) + " has ip=" +
                         std::to_string(a) + " in=" + std::to_string(b));
    if (b > 0) {
      if (seg_of[a - 1] != seg_of[b - 1])
        return set_err(c, SOLV_GPU_BAD_INPUT,
                       "matrix_set_batch: face " + std::to_string(f + 1) + " couples two systems");
      deg[a - 1]++;
      deg[b - 1]++;
      if (b < a) orient = false;
    }
  }
  std::vector<long long> rp(N + 1, 0);
  for (int i = 0; i < N; ++i) rp[i + 1] = rp[i] + deg[i];
  // rows in caller numbering, faces ascending (grd_conn.f90:129-152)
  std::vector<int> rnb(rp[N]), rsrc(rp[N]);
  std::vector<long long> fill(rp.begin(), rp.end() - 1);
  for (int f = 0; f < F; ++f) {
    int a = ip[f] - 1, b = in[f] - 1;
    if (b < 0) continue;
    rnb[fill[a]] = b;
    rsrc[fill[a]++] = 2 * f;
    rnb[fill[b]] = a;
    rsrc[fill[b]++] = 2 * f + 1;
  }
  // wavefront levels of the lower DAG (neighbour index below the cell)
  std::vector<int> lev(N, 0);
  int nl = 0;
  for (int i = 0; i < N; ++i) {
    int l = 0;
    for (long long k = rp[i]; k < rp[i + 1]; ++k)
      if (rnb[k] < i) l = std::max(l, lev[rnb[k]] + 1);
    lev[i] = l;
    nl = std::max(nl, l + 1);
  }
  // internal order: system-major, then level, then caller order, so each
  // system is one contiguous range (reductions) and, for one system, each
  // level is one contiguous range (sweeps)
  std::vector<int> old_of_new(N), new_of_old(N);
  std::vector<int> seg_c0(nsys), seg_c1(nsys);
  {
    std::vector<long long> key(N);
    std::vector<int> cnt((size_t)nsys * nl + 1, 0);
    for (int i = 0; i < N; ++i) cnt[(size_t)seg_of[i] * nl + lev[i] + 1]++;
    for (size_t k = 0; k + 1 < cnt.size(); ++k) cnt[k + 1] += cnt[k];
    std::vector<int> pos(cnt.begin(), cnt.end() - 1);
    for (int i = 0; i < N; ++i) {
      int k = pos[(size_t)seg_of[i] * nl + lev[i]]++;
      old_of_new[k] = i;
      new_of_old[i] = k;
    }
    for (int k = 0; k < nsys; ++k) {
      seg_c0[k] = cnt[(size_t)k * nl];
      seg_c1[k] = cnt[(size_t)(k + 1) * nl];
    }
  }
  // cells per level (the sweep depth reported in the statistics)
  std::vector<int> lcnt(nl + 1, 0);
  for (int i = 0; i < N; ++i) lcnt[lev[i] + 1]++;
  for (int l = 0; l < nl; ++l) lcnt[l + 1] += lcnt[l];
  c->lvl_ptr.assign(lcnt.begin(), lcnt.end());
  // sliced ELL, 32 cells per slice
  const int ns = (N + 31) / 32;
  std::vector<int> sp(ns + 1, 0);
  std::vector<uint8_t> sw(ns, 0);
  long long total = 0;
  for (int s = 0; s < ns; ++s) {
    int w = 0;
    for (int l = 0; l < 32; ++l) {
      int i = s * 32 + l;
      if (i < N) w = std::max(w, deg[old_of_new[i]]);
    }
    if (w > 255) return set_err(c, SOLV_GPU_BAD_INPUT, "matrix_set: a cell has more than 255 faces");
    sw[s] = (uint8_t)w;
    if (total > (1LL << 31) - 1 - 32LL * w)
      return set_err(c, SOLV_GPU_BAD_INPUT, "matrix_set: too many matrix entries for int32 offsets");
    sp[s] = (int)total;
    total += 32LL * w;
  }
  sp[ns] = (int)total;
  std::vector<int> hcol(total, -1), hsrc(total, -1);
  for (int s = 0; s < ns; ++s)
    for (int l = 0; l < 32; ++l) {
      int i = s * 32 + l;
      if (i >= N) continue;
      int o = old_of_new[i];
      int k = 0;
      for (long long q = rp[o]; q < rp[o + 1]; ++q, ++k) {
        long long e = sp[s] + (long long)k * 32 + l;
        hcol[e] = new_of_old[rnb[q]];
        hsrc[e] = rsrc[q];
      }
    }
  drop_graphs(c);
  c->N = N;
  c->F = F;
  c->n_seg = nsys;
  c->t_ready = c->tf_ready = false;
  c->orient_std = orient;
  c->n_slots = total;
  c->n_slice = ns;
  c->f32_valid = false;
  c->g_feat_valid = false;
  c->mg_valid = false;
  c->mg.clear();
  c->pcg_local.clear();
  cudaStream_t st = c->stream;
  CUDA_TRY(c, c->old_of_new.ensure(N * sizeof(int)));
  CUDA_TRY(c, c->slice_ptr.ensure((ns + 1) * sizeof(int)));
  CUDA_TRY(c, c->slice_w.ensure(ns));
  CUDA_TRY(c, c->col.ensure(total * sizeof(int)));
  CUDA_TRY(c, c->slot_src.ensure(total * sizeof(int)));
  CUDA_TRY(c, c->val.ensure(total * sizeof(double)));
  if (!orient) CUDA_TRY(c, c->sval.ensure(total * sizeof(double)));
  CUDA_TRY(c, c->diag.ensure(N * sizeof(double)));
  CUDA_TRY(c, c->fp.ensure(std::max(F, 1) * sizeof(double)));
  CUDA_TRY(c, c->fn.ensure(std::max(F, 1) * sizeof(double)));
  CUDA_TRY(c, cudaMemcpyAsync(c->old_of_new.p, old_of_new.data(), N * sizeof(int), cudaMemcpyHostToDevice, st));
  CUDA_TRY(c, cudaMemcpyAsync(c->slice_ptr.p, sp.data(), (ns + 1) * sizeof(int), cudaMemcpyHostToDevice, st));
  CUDA_TRY(c, cudaMemcpyAsync(c->slice_w.p, sw.data(), ns, cudaMemcpyHostToDevice, st));
  CUDA_TRY(c, cudaMemcpyAsync(c->col.p, hcol.data(), total * sizeof(int), cudaMemcpyHostToDevice, st));
  CUDA_TRY(c, cudaMemcpyAsync(c->slot_src.p, hsrc.data(), total * sizeof(int), cudaMemcpyHostToDevice, st));
  CUDA_TRY(c, cudaStreamSynchronize(st));  // host vectors die here
  c->seg_c0_caller.assign(seg_c0.begin(), seg_c0.end());
  c->seg_c1_caller.assign(seg_c1.begin(), seg_c1.end());
  int rc = build_segments(c, seg_c0, seg_c1);
  if (rc) return rc;
  c->has_matrix = true;
  return SOLV_GPU_OK;
}

int matrix_values_dev(solv_gpu_ctx* c, const double* p, const double* n, const double* pl) {
  if (!c->has_matrix) return set_err(c, SOLV_GPU_NO_MATRIX, "no matrix set");
  const int N = c->N;
  if (p != c->fp.as<double>() && c->F > 0)
    CUDA_TRY(c, cudaMemcpyAsync(c->fp.p, p, c->F * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  if (n != c->fn.as<double>() && c->F > 0)
    CUDA_TRY(c, cudaMemcpyAsync(c->fn.p, n, c->F * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  sg::k_fill_values<double><<<grid_for(c, N), c->block, 0, c->stream>>>(
      N, c->slice_ptr.as<int>(), c->slice_w.as<uint8_t>(), c->slot_src.as<int>(),
      c->col.as<int>(), c->fp.as<double>(), c->fn.as<double>(), c->val.as<double>(),
      c->orient_std ? nullptr : c->sval.as<double>());
  sg::k_fill_diag<double><<<grid_for(c, N), c->block, 0, c->stream>>>(
      N, c->old_of_new.as<int>(), pl, c->diag.as<double>());
  CUDA_TRY(c, cudaGetLastError());
  c->f32_valid = false;
  c->g_feat_valid = false;
  return SOLV_GPU_OK;
}

int ensure_f32_matrix(solv_gpu_ctx* c) {
  if (c->f32_valid) return SOLV_GPU_OK;
  CUDA_TRY(c, c->valf.ensure(c->n_slots * sizeof(float)));
  CUDA_TRY(c, c->diagf.ensure(c->N * sizeof(float)));
  sg::k_convert<double, float><<<grid_for(c, c->n_slots), c->block, 0, c->stream>>>(
      c->n_slots, c->val.as<double>(), c->valf.as<float>());
  if (!c->orient_std) {
    CUDA_TRY(c, c->svalf.ensure(c->n_slots * sizeof(float)));
    sg::k_convert<double, float><<<grid_for(c, c->n_slots), c->block, 0, c->stream>>>(
        c->n_slots, c->sval.as<double>(), c->svalf.as<float>());
  }
  sg::k_rowsum_diag<<<grid_for(c, c->N), c->block, 0, c->stream>>>(c->N, rows<double>(c),
                                                                   c->diagf.as<float>());
  CUDA_TRY(c, cudaGetLastError());
  c->f32_valid = true;
  return SOLV_GPU_OK;
}

// ---- learned preconditioner ------------------------------------------------------
gnn::Feat gnn_feat(solv_gpu_ctx* c) {
  gnn::Feat F;
  F.rsd = c->g_rsd.as<float>();
  F.frs = c->g_frs.as<float>();
  F.fdeg = c->g_fdeg.as<float>();
  F.gw = c->g_gw.as<float>();
  return F;
}

int gnn_grid_warps(solv_gpu_ctx* c, long long n_threads) {
  long long g = (n_threads + 255) / 256;
  return (int)std::max(1LL, std::min(g, (long long)c->n_sm * 16));
}

// Features of the current matrix, packed BF16 weights and inference buffers.
int gnn_prepare(solv_gpu_ctx* c) {
  if (!c->g_has_params)
    return set_err(c, SOLV_GPU_BAD_INPUT, "learned preconditioner: no parameters set");
  if (c->n_seg != 1) return set_err(c, SOLV_GPU_BAD_INPUT, "learned preconditioner: one system only");
  int rc = ensure_f32_matrix(c);
  if (rc) return rc;
  const int N = c->N;
  const void* before[6] = {c->g_h0.p, c->g_h1.p, c->g_u.p, c->g_wcat.p, c->g_q.p, c->g_ge.p};
  if (!c->g_feat_valid) {
    CUDA_TRY(c, c->g_rsd.ensure(N * sizeof(float)));
    CUDA_TRY(c, c->g_frs.ensure(N * sizeof(float)));
    CUDA_TRY(c, c->g_fdeg.ensure(N * sizeof(float)));
    CUDA_TRY(c, c->g_gw.ensure(c->n_slots * sizeof(float)));
    gnn::k_gnn_features<<<grid_for(c, N), c->block, 0, c->stream>>>(
        N, rows<double>(c), c->g_rsd.as<float>(), c->g_frs.as<float>(), c->g_fdeg.as<float>(),
        c->g_gw.as<float>());
    CUDA_TRY(c, cudaGetLastError());
    c->g_feat_valid = true;
  }
  if (!c->g_wcat_valid) {
    const int nw = gnn::NL * 2 * gnn::H * gnn::H;
    CUDA_TRY(c, c->g_wcat.ensure(nw * sizeof(__nv_bfloat16)));
    gnn::k_gnn_pack<<<(nw + 255) / 256, 256, 0, c->stream>>>(c->g_param.as<float>(),
                                                             c->g_wcat.as<__nv_bfloat16>());
    CUDA_TRY(c, cudaGetLastError());
    c->g_wcat_valid = true;
  }
  CUDA_TRY(c, c->g_h0.ensure((size_t)N * gnn::H * sizeof(__nv_bfloat16)));
  CUDA_TRY(c, c->g_h1.ensure((size_t)N * gnn::H * sizeof(__nv_bfloat16)));
  CUDA_TRY(c, c->g_u.ensure((size_t)N * sizeof(float)));
  CUDA_TRY(c, c->g_q.ensure((size_t)N * sizeof(float)));
  CUDA_TRY(c, c->g_he.ensure((size_t)N * sizeof(float)));
  CUDA_TRY(c, c->g_ge.ensure((size_t)c->n_slots * sizeof(float)));
  const void* after[6] = {c->g_h0.p, c->g_h1.p, c->g_u.p, c->g_wcat.p, c->g_q.p, c->g_ge.p};
  for (int k = 0; k < 6; ++k)
    if (before[k] != after[k]) drop_graphs(c);
  return SOLV_GPU_OK;
}

// Build the preconditioner for this solve from the initial residual r0
// (internal order; its scale gs already in lane 0): the network on the
// tensor cores, then the heads (q = s / sqrt(d)) and the face weights gE.
template <typename T>
void gnn_build(solv_gpu_ctx* c, const T* r0) {
  const int N = c->N;
  gnn::Feat F = gnn_feat(c);
  const float* P = c->g_param.as<float>();
  __nv_bfloat16* h0 = c->g_h0.as<__nv_bfloat16>();
  __nv_bfloat16* h1 = c->g_h1.as<__nv_bfloat16>();
  gnn::k_gnn_enc<T><<<gnn_grid_warps(c, (long long)N * 32), 256, 0, c->stream>>>(
      N, F, r0, P, c->lanes.as<Lane>(), h0, c->g_u.as<float>());
  const int tiles = (N + gnn::TC_CELLS - 1) / gnn::TC_CELLS;
  if (c->gnn_layer_blocks <= 0) {  // resident blocks per SM of the layer kernel
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gnn::k_gnn_layer_tc,
                                                      gnn::TC_WARPS * 32, 0) != cudaSuccess ||
        per_sm < 1)
      per_sm = 8;
    c->gnn_layer_blocks = per_sm;
  }
  const int tcb = std::max(1, std::min((tiles + gnn::TC_WARPS - 1) / gnn::TC_WARPS,
                                       c->n_sm * c->gnn_layer_blocks));
  __nv_bfloat16 *hin = h0, *hout = h1;
  for (int l = 0; l < gnn::NL; ++l) {
    gnn::k_gnn_layer_tc<<<tcb, gnn::TC_WARPS * 32, 0, c->stream>>>(
        N, rows<float>(c), F, hin, hout, c->g_wcat.as<__nv_bfloat16>() + l * 2 * gnn::H * gnn::H,
        P + gnn::P_LAYER + l * gnn::LAYER_SZ + 2 * gnn::H * gnn::H);
    std::swap(hin, hout);
  }
  gnn::k_gnn_heads<__nv_bfloat16><<<grid_for(c, N), 256, 0, c->stream>>>(
      N, hin, P, c->g_rsd.as<float>(), nullptr, c->g_q.as<float>(), c->g_he.as<float>());
  gnn::k_gnn_edges<<<grid_for(c, N), c->block, 0, c->stream>>>(
      N, rows<float>(c), F, c->g_he.as<float>(), P, nullptr, c->g_ge.as<float>());
  c->launches += 3 + gnn::NL;
}

// ---- aggregation multigrid (mg.cuh) -----------------------------------------------
template <typename V>
cudaError_t upload(DevBuf& d, const std::vector<V>& h, cudaStream_t s) {
  cudaError_t e = d.ensure(std::max<size_t>(h.size(), 1) * sizeof(V));
  if (e != cudaSuccess || h.empty()) return e;
  return cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(V), cudaMemcpyHostToDevice, s);
}

// ---- the hierarchy built on the GPU (mg_build.cuh) ------------------------------
// Exclusive prefix sum out[0..n] of in[0..n); the total (out[n]) also to
// *total_host when that is given (a synchronising copy).
int dev_scan(solv_gpu_ctx* c, const int* in, int* out, int n, DevBuf& bs, int* total_host) {
  cudaStream_t s = c->stream;
  if (n <= 0) {
    CUDA_TRY(c, cudaMemsetAsync(out, 0, sizeof(int), s));
    if (total_host) *total_host = 0;
    return SOLV_GPU_OK;
  }
  const int nb = (n + mgb::kScanBlock - 1) / mgb::kScanBlock;
  CUDA_TRY(c, bs.ensure((size_t)(nb + 1) * sizeof(int)));
  int* b = bs.as<int>();
  mgb::k_scan_block<<<nb, mgb::kScanBlock, 0, s>>>(n, in, out, b);
  mgb::k_scan_sums<<<1, mgb::kScanBlock, 0, s>>>(nb, b, b + nb);
  mgb::k_scan_add<<<(n + 256) / 256, 256, 0, s>>>(n, out, b, b + nb);
  CUDA_TRY(c, cudaGetLastError());
  if (total_host) {
    CUDA_TRY(c, cudaMemcpyAsync(total_host, out + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(c, cudaStreamSynchronize(s));
  }
  return SOLV_GPU_OK;
}

// A coarse level's structure as the GPU Galerkin walk builds it.
struct CoarseDev {
  int nc = 0;
  int n_slots = 0;
  DevBuf sp, sw, col, gptr, gsrc, mptr, cells;
};

// Members of the nc aggregates of agg (sorted lists) and the Galerkin
// structure of the coarse level over the finer level f (n cells).  Returns
// SOLV_GPU_TOO_LARGE when a coarse row would exceed 255 slots.
int gpu_galerkin(solv_gpu_ctx* c, mgb::Ell f, int n, const int* agg, int nc, CoarseDev& C) {
  cudaStream_t s = c->stream;
  const int B = 256;
  const int G = grid_for(c, std::max(n, nc));
  DevBuf cnt, cur, deg, slots, bs, err;
  C.nc = nc;
  CUDA_TRY(c, cnt.ensure((size_t)nc * sizeof(int)));
  CUDA_TRY(c, cur.ensure((size_t)nc * sizeof(int)));
  CUDA_TRY(c, C.mptr.ensure((size_t)(nc + 1) * sizeof(int)));
  CUDA_TRY(c, C.cells.ensure((size_t)n * sizeof(int)));
  CUDA_TRY(c, cudaMemsetAsync(cnt.p, 0, (size_t)nc * sizeof(int), s));
  CUDA_TRY(c, cudaMemsetAsync(cur.p, 0, (size_t)nc * sizeof(int), s));
  mgb::k_count<<<G, B, 0, s>>>(n, agg, cnt.as<int>());
  int rc = dev_scan(c, cnt.as<int>(), C.mptr.as<int>(), nc, bs, nullptr);
  if (rc) return rc;
  mgb::k_place<<<G, B, 0, s>>>(n, agg, C.mptr.as<int>(), cur.as<int>(), C.cells.as<int>());
  mgb::k_sort_members<<<grid_for(c, nc), B, 0, s>>>(nc, C.mptr.as<int>(), C.cells.as<int>());
  CUDA_TRY(c, err.ensure(sizeof(int)));
  CUDA_TRY(c, cudaMemsetAsync(err.p, 0, sizeof(int), s));
  CUDA_TRY(c, deg.ensure((size_t)nc * sizeof(int)));
  const int gw = (int)std::max(1LL, std::min<long long>((nc + mgb::kGalWarps - 1) / mgb::kGalWarps,
                                                        (long long)c->n_sm * 8));
  mgb::k_galerkin<0><<<gw, mgb::kGalWarps * 32, 0, s>>>(
      nc, f, agg, C.mptr.as<int>(), C.cells.as<int>(), deg.as<int>(), nullptr, nullptr, nullptr,
      nullptr, nullptr, err.as<int>());
  int herr = 0;
  CUDA_TRY(c, cudaMemcpyAsync(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(c, cudaStreamSynchronize(s));
  if (herr) return SOLV_GPU_TOO_LARGE;
  const int ns = (nc + 31) / 32;
  CUDA_TRY(c, C.sw.ensure(std::max(ns, 1)));
  CUDA_TRY(c, slots.ensure((size_t)std::max(ns, 1) * sizeof(int)));
  CUDA_TRY(c, C.sp.ensure((size_t)(ns + 1) * sizeof(int)));
  mgb::k_slice_widths<<<grid_for(c, ns), B, 0, s>>>(nc, deg.as<int>(), C.sw.as<uint8_t>(),
                                                   slots.as<int>());
  int total = 0;
  if ((rc = dev_scan(c, slots.as<int>(), C.sp.as<int>(), ns, bs, &total))) return rc;
  if (total < 0) return SOLV_GPU_TOO_LARGE;  // beyond int32 slot offsets
  C.n_slots = total;
  CUDA_TRY(c, C.col.ensure((size_t)std::max(total, 1) * sizeof(int)));
  CUDA_TRY(c, cnt.ensure((size_t)std::max(total, 1) * sizeof(int)));
  CUDA_TRY(c, cudaMemsetAsync(C.col.p, 0xff, (size_t)std::max(total, 1) * sizeof(int), s));
  CUDA_TRY(c, cudaMemsetAsync(cnt.p, 0, (size_t)std::max(total, 1) * sizeof(int), s));
  mgb::k_galerkin<1><<<gw, mgb::kGalWarps * 32, 0, s>>>(
      nc, f, agg, C.mptr.as<int>(), C.cells.as<int>(), nullptr, C.sp.as<int>(), C.col.as<int>(),
      cnt.as<int>(), nullptr, nullptr, err.as<int>());
  CUDA_TRY(c, C.gptr.ensure((size_t)(total + 1) * sizeof(int)));
  int n_src = 0;
  if ((rc = dev_scan(c, cnt.as<int>(), C.gptr.as<int>(), total, bs, &n_src))) return rc;
  CUDA_TRY(c, C.gsrc.ensure((size_t)std::max(n_src, 1) * sizeof(int)));
  mgb::k_galerkin<2><<<gw, mgb::kGalWarps * 32, 0, s>>>(
      nc, f, agg, C.mptr.as<int>(), C.cells.as<int>(), nullptr, C.sp.as<int>(), nullptr, nullptr,
      C.gptr.as<int>(), C.gsrc.as<int>(), err.as<int>());
  CUDA_TRY(c, cudaGetLastError());
  CUDA_TRY(c, cudaStreamSynchronize(s));  // before the local buffers are freed
  return SOLV_GPU_OK;
}

// Aggregation of one level (n cells, structure g, strengths w) into
// agg (n entries) and *nc aggregates: passes of handshake matching on the
// pass graphs, then the singletons joined to a neighbour's aggregate.
int gpu_aggregate(solv_gpu_ctx* c, mgb::Ell g, const float* w, int n, int passes, DevBuf& agg,
                  int* nc_out) {
  cudaStream_t s = c->stream;
  const int B = 256;
  DevBuf mate, prop, flag, id, aggp, bs, size, used, rep;
  CoarseDev P;       // the current pass graph (after the first pass)
  DevBuf pw, pw2;    // its strengths
  CUDA_TRY(c, agg.ensure((size_t)n * sizeof(int)));
  mgb::Ell gp = g;
  const float* wp = w;
  int np = n;
  for (int p = 0; p < passes; ++p) {
    const int G = grid_for(c, np);
    CUDA_TRY(c, mate.ensure((size_t)np * sizeof(int)));
    CUDA_TRY(c, prop.ensure((size_t)np * sizeof(int)));
    CUDA_TRY(c, flag.ensure((size_t)np * sizeof(int)));
    CUDA_TRY(c, id.ensure((size_t)(np + 1) * sizeof(int)));
    CUDA_TRY(c, aggp.ensure((size_t)np * sizeof(int)));
    CUDA_TRY(c, cudaMemsetAsync(mate.p, 0xff, (size_t)np * sizeof(int), s));
    for (int r = 0; r < mgb::kRounds; ++r) {
      mgb::k_hs_propose<<<G, B, 0, s>>>(np, gp, wp, mate.as<int>(), prop.as<int>());
      mgb::k_hs_accept<<<G, B, 0, s>>>(np, prop.as<int>(), mate.as<int>());
    }
    CUDA_TRY(c, rep.ensure((size_t)np * sizeof(int)));
    // nodes the handshakes left alone stay alone for this pass, unless the
    // pass would then keep more than 3/4 of its nodes: then they join a pair
    int nn = 0, rc = 0;
    for (int join = 0; join < 2; ++join) {
      mgb::k_hs_rep<<<G, B, 0, s>>>(np, gp, wp, mate.as<int>(), join, rep.as<int>(), flag.as<int>());
      if ((rc = dev_scan(c, flag.as<int>(), id.as<int>(), np, bs, &nn))) return rc;
      if (nn <= 0.75 * np) break;
    }
    mgb::k_hs_number<<<G, B, 0, s>>>(np, rep.as<int>(), id.as<int>(), aggp.as<int>());
    if (p == 0)
      CUDA_TRY(c, cudaMemcpyAsync(agg.p, aggp.p, (size_t)n * sizeof(int), cudaMemcpyDeviceToDevice, s));
    else
      mgb::k_compose<<<grid_for(c, n), B, 0, s>>>(n, agg.as<int>(), aggp.as<int>());
    if (p + 1 < passes && nn < np) {  // the next pass graph and its strengths
      CoarseDev Q;
      if ((rc = gpu_galerkin(c, gp, np, aggp.as<int>(), nn, Q))) {
        if (rc != SOLV_GPU_TOO_LARGE) return rc;
        np = nn;  // a pass graph too dense for 255 slots a row: pair no further
        break;
      }
      CUDA_TRY(c, pw2.ensure((size_t)std::max(Q.n_slots, 1) * sizeof(float)));
      mgb::k_sum_abs<<<grid_for(c, Q.n_slots), B, 0, s>>>(Q.n_slots, Q.gptr.as<int>(),
                                                           Q.gsrc.as<int>(), wp, pw2.as<float>());
      CUDA_TRY(c, cudaStreamSynchronize(s));  // the old pass graph is freed below
      P.sp.swap(Q.sp);
      P.sw.swap(Q.sw);
      P.col.swap(Q.col);
      P.n_slots = Q.n_slots;
      pw.swap(pw2);
      gp.sp = P.sp.as<int>();
      gp.sw = P.sw.as<uint8_t>();
      gp.col = P.col.as<int>();
      wp = pw.as<float>();
    }
    np = nn;
    if (nn == 0) break;
  }
  // singletons join a neighbour's aggregate; dense renumbering
  const int G = grid_for(c, n);
  CUDA_TRY(c, size.ensure((size_t)np * sizeof(int)));
  CUDA_TRY(c, used.ensure((size_t)np * sizeof(int)));
  CUDA_TRY(c, id.ensure((size_t)(np + 1) * sizeof(int)));
  CUDA_TRY(c, aggp.ensure((size_t)n * sizeof(int)));
  CUDA_TRY(c, cudaMemsetAsync(size.p, 0, (size_t)np * sizeof(int), s));
  CUDA_TRY(c, cudaMemsetAsync(used.p, 0, (size_t)np * sizeof(int), s));
  mgb::k_count<<<G, B, 0, s>>>(n, agg.as<int>(), size.as<int>());
  mgb::k_join_singletons<<<G, B, 0, s>>>(n, g, w, agg.as<int>(), size.as<int>(), aggp.as<int>());
  mgb::k_mark<<<G, B, 0, s>>>(n, aggp.as<int>(), used.as<int>());
  int nc = 0;
  int rc = dev_scan(c, used.as<int>(), id.as<int>(), np, bs, &nc);
  if (rc) return rc;
  mgb::k_renumber<<<G, B, 0, s>>>(n, aggp.as<int>(), id.as<int>());
  agg.swap(aggp);
  CUDA_TRY(c, cudaGetLastError());
  CUDA_TRY(c, cudaStreamSynchronize(s));  // before the local buffers are freed
  *nc_out = nc;
  return SOLV_GPU_OK;
}

// The hierarchy for the current structure, built on the GPU from the
// coefficients present now.  Same rules and stopping tests as the host
// build below.
int mg_setup_gpu(solv_gpu_ctx* c, std::vector<std::unique_ptr<MgLevel>>& levels, bool& ok) {
  cudaStream_t s = c->stream;
  const int B = c->block;
  int n = c->N;
  mgb::Ell g{c->slice_ptr.as<int>(), c->slice_w.as<uint8_t>(), c->col.as<int>()};
  DevBuf w0, wn;
  CUDA_TRY(c, w0.ensure((size_t)std::max<long long>(c->n_slots, 1) * sizeof(float)));
  mgb::k_abs<<<grid_for(c, c->n_slots), B, 0, s>>>(c->n_slots, c->valf.as<float>(), w0.as<float>());
  const float* w = w0.as<float>();
  const float* vprev = c->valf.as<float>();
  ok = n > mg::kCoarsest;
  while (ok && n > mg::kCoarsest) {
    if ((int)levels.size() >= std::min(c->mg_max_levels, mg::kMaxLevels)) { ok = false; break; }
    auto L = std::make_unique<MgLevel>();
    int nc = 0;
    int rc = gpu_aggregate(c, g, w, n, 3, L->agg_of, &nc);
    if (rc) return rc;
    if (nc > 0.75 * n || nc < 1) { ok = false; break; }  // coarsening stalled
    CoarseDev C;
    rc = gpu_galerkin(c, g, n, L->agg_of.as<int>(), nc, C);
    if (rc == SOLV_GPU_TOO_LARGE) { ok = false; break; }
    if (rc) return rc;
    L->n = nc;
    L->n_slots = C.n_slots;
    L->slice_ptr.swap(C.sp);
    L->slice_w.swap(C.sw);
    L->col.swap(C.col);
    L->gptr.swap(C.gptr);
    L->gsrc.swap(C.gsrc);
    L->agg_ptr.swap(C.mptr);
    L->agg_cells.swap(C.cells);
    const size_t vb = (size_t)nc * sizeof(float);
    CUDA_TRY(c, L->val.ensure((size_t)std::max(C.n_slots, 1) * sizeof(float)));
    CUDA_TRY(c, L->rs.ensure(vb));
    CUDA_TRY(c, L->dinv.ensure(vb));
    CUDA_TRY(c, L->x.ensure(vb));
    CUDA_TRY(c, L->b.ensure(vb));
    CUDA_TRY(c, L->t.ensure(vb));
    CUDA_TRY(c, L->y.ensure(vb));
    // coarse coefficients now: the next aggregation's strengths
    mg::k_mg_gather_slots<<<grid_for(c, C.n_slots), B, 0, s>>>(
        C.n_slots, L->gptr.as<int>(), L->gsrc.as<int>(), vprev, L->val.as<float>());
    CUDA_TRY(c, wn.ensure((size_t)std::max(C.n_slots, 1) * sizeof(float)));
    mgb::k_abs<<<grid_for(c, C.n_slots), B, 0, s>>>(C.n_slots, L->val.as<float>(), wn.as<float>());
    CUDA_TRY(c, cudaGetLastError());
    w0.swap(wn);
    w = w0.as<float>();
    vprev = L->val.as<float>();
    g = mgb::Ell{L->slice_ptr.as<int>(), L->slice_w.as<uint8_t>(), L->col.as<int>()};
    n = nc;
    levels.push_back(std::move(L));
  }
  CUDA_TRY(c, cudaStreamSynchronize(s));
  return SOLV_GPU_OK;
}

// Build the hierarchy for the current structure from the coefficients
// present now (once per structure): on the GPU (mg_build.cuh, the default)
// or with the host aggregation (SOLV_OPT_MG_BUILD 1).  A hierarchy that
// cannot reach kCoarsest cells (coarsening stalls) is not used: the solve
// then runs with the one-level preconditioner.
int mg_setup(solv_gpu_ctx* c) {
  if (c->mg_valid && c->mg_built_max == c->mg_max_levels) return SOLV_GPU_OK;
  c->mg_built_max = c->mg_max_levels;
  auto t0 = std::chrono::steady_clock::now();
  int rc = ensure_f32_matrix(c);
  if (rc) return rc;
  drop_graphs(c);
  c->mg.clear();
  cudaStream_t s = c->stream;
  if (c->mg_build == 0) {
    std::vector<std::unique_ptr<MgLevel>> levels;
    bool ok = true;
    if ((rc = mg_setup_gpu(c, levels, ok))) return rc;
    c->mg_valid = true;
    if (ok && !levels.empty()) {
      c->mg = std::move(levels);
      const int nL = c->mg.back()->n;
      CUDA_TRY(c, c->mg_x0.ensure((size_t)c->N * sizeof(float)));
      CUDA_TRY(c, c->mg_t0.ensure((size_t)c->N * sizeof(float)));
      CUDA_TRY(c, c->mg_dinv0.ensure((size_t)c->N * sizeof(float)));
      CUDA_TRY(c, c->mg_dq.ensure((size_t)c->N * sizeof(float)));
      CUDA_TRY(c, c->mg_dense.ensure((size_t)nL * nL * sizeof(double)));
      CUDA_TRY(c, c->mg_ainv.ensure((size_t)nL * nL * sizeof(float)));
    }
    c->mg_setup_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return SOLV_GPU_OK;
  }
  // host build: level 0 from the device
  int n = c->N;
  const int ns0 = c->n_slice;
  std::vector<int> sp(ns0 + 1), col(c->n_slots);
  std::vector<uint8_t> sw(ns0);
  std::vector<float> val(c->n_slots), rs(n);
  CUDA_TRY(c, cudaMemcpyAsync(sp.data(), c->slice_ptr.p, (ns0 + 1) * sizeof(int), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(c, cudaMemcpyAsync(sw.data(), c->slice_w.p, ns0, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(c, cudaMemcpyAsync(col.data(), c->col.p, c->n_slots * sizeof(int), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(c, cudaMemcpyAsync(val.data(), c->valf.p, c->n_slots * sizeof(float), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(c, cudaStreamSynchronize(s));
  std::vector<std::unique_ptr<MgLevel>> levels;
  bool ok = n > mg::kCoarsest;
  while (ok && n > mg::kCoarsest) {
    if ((int)levels.size() >= std::min(c->mg_max_levels, mg::kMaxLevels)) { ok = false; break; }
    mg::Graph g = mg::graph_of(n, sp, sw, col, val);
    std::vector<int> agg;
    const int nc = mg::aggregate(g, 3, agg);
    if (nc > 0.75 * n) { ok = false; break; }  // coarsening stalled
    mg::CoarseHost C;
    if (!mg::build_coarse(n, sp, sw, col, agg, nc, C)) { ok = false; break; }
    // coarse coefficients on the host too (the next aggregation's strengths)
    std::vector<float> cval(C.n_slots, 0.0f);
    for (long long e = 0; e < C.n_slots; ++e) {
      double a = 0.0;
      for (int k = C.gptr[e]; k < C.gptr[e + 1]; ++k) a += val[C.gsrc[k]];
      cval[e] = (float)a;
    }
    auto L = std::make_unique<MgLevel>();
    L->n = nc;
    L->n_slots = C.n_slots;
    CUDA_TRY(c, upload(L->slice_ptr, C.slice_ptr, s));
    CUDA_TRY(c, upload(L->slice_w, C.slice_w, s));
    CUDA_TRY(c, upload(L->col, C.col, s));
    CUDA_TRY(c, upload(L->gptr, C.gptr, s));
    CUDA_TRY(c, upload(L->gsrc, C.gsrc, s));
    CUDA_TRY(c, upload(L->agg_ptr, C.agg_ptr, s));
    CUDA_TRY(c, upload(L->agg_cells, C.agg_cells, s));
    CUDA_TRY(c, upload(L->agg_of, C.agg_of, s));
    const size_t vb = (size_t)nc * sizeof(float);
    CUDA_TRY(c, L->val.ensure(std::max<long long>(C.n_slots, 1) * sizeof(float)));
    CUDA_TRY(c, L->rs.ensure(vb));
    CUDA_TRY(c, L->dinv.ensure(vb));
    CUDA_TRY(c, L->x.ensure(vb));
    CUDA_TRY(c, L->b.ensure(vb));
    CUDA_TRY(c, L->t.ensure(vb));
    CUDA_TRY(c, L->y.ensure(vb));
    CUDA_TRY(c, cudaStreamSynchronize(s));  // host arrays die below
    levels.push_back(std::move(L));
    sp.swap(C.slice_ptr);
    sw.swap(C.slice_w);
    col.swap(C.col);
    val.swap(cval);
    n = nc;
  }
  c->mg_valid = true;
  if (!ok || levels.empty()) {
    c->mg.clear();
    c->mg_setup_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return SOLV_GPU_OK;
  }
  c->mg = std::move(levels);
  const int nL = c->mg.back()->n;
  CUDA_TRY(c, c->mg_x0.ensure((size_t)c->N * sizeof(float)));
  CUDA_TRY(c, c->mg_t0.ensure((size_t)c->N * sizeof(float)));
  CUDA_TRY(c, c->mg_dinv0.ensure((size_t)c->N * sizeof(float)));
  CUDA_TRY(c, c->mg_dq.ensure((size_t)c->N * sizeof(float)));
  CUDA_TRY(c, c->mg_dense.ensure((size_t)nL * nL * sizeof(double)));
  CUDA_TRY(c, c->mg_ainv.ensure((size_t)nL * nL * sizeof(float)));
  c->mg_setup_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return SOLV_GPU_OK;
}

// Coefficients of every coarse level for the current values (each solve):
// Galerkin sums level by level, inverse diagonals, the coarsest inverse.
int mg_values(solv_gpu_ctx* c) {
  int rc = ensure_f32_matrix(c);
  if (rc) return rc;
  cudaStream_t s = c->stream;
  const int B = c->block;
  mg::k_mg_dinv<<<grid_for(c, c->N), B, 0, s>>>(c->N, rows<float>(c), c->mg_dinv0.as<float>());
  const float* vprev = c->valf.as<float>();
  const float* rsprev = c->diagf.as<float>();
  for (auto& L : c->mg) {
    mg::k_mg_gather_slots<<<grid_for(c, L->n_slots), B, 0, s>>>(
        L->n_slots, L->gptr.as<int>(), L->gsrc.as<int>(), vprev, L->val.as<float>());
    mg::k_mg_rowsum<<<grid_for(c, L->n), B, 0, s>>>(L->n, L->agg_ptr.as<int>(),
                                                    L->agg_cells.as<int>(), rsprev, L->rs.as<float>());
    mg::k_mg_dinv<<<grid_for(c, L->n), B, 0, s>>>(L->n, L->rows(), L->dinv.as<float>());
    vprev = L->val.as<float>();
    rsprev = L->rs.as<float>();
  }
  MgLevel& C = *c->mg.back();
  mg::k_mg_dense<<<grid_for(c, C.n), B, 0, s>>>(C.n, C.rows(), c->mg_dense.as<double>());
  mg::k_mg_invert<<<1, 1024, 0, s>>>(C.n, c->mg_dense.as<double>(), c->mg_ainv.as<float>());
  c->launches += 2 + 3 * (int)c->mg.size() + 2;
  CUDA_TRY(c, cudaGetLastError());
  return SOLV_GPU_OK;
}

// The V-cycle below level 0: level 1's right-hand side mg[0]->b in, its
// correction mg[0]->y out.  Returns the number of kernels launched.
int mg_coarse_cycle(solv_gpu_ctx* c, const int* na) {
  cudaStream_t s = c->stream;
  const int B = c->block;
  const float w = (float)c->mg_omega, a = (float)c->mg_alpha;
  const int L = (int)c->mg.size();
  int k = 0;
  for (int l = 0; l + 1 < L; ++l) {
    MgLevel& F = *c->mg[l];
    MgLevel& C = *c->mg[l + 1];
    with_chunk(c->row_chunk, [&](auto ch) {
      mg::k_mg_pre<decltype(ch)::value><<<grid_for(c, F.n), B, 0, s>>>(
          F.n, F.rows(), F.dinv.as<float>(), w, F.b.as<float>(), F.x.as<float>(), F.t.as<float>(),
          na);
    });
    mg::k_mg_restrict<<<grid_for(c, C.n), B, 0, s>>>(C.n, C.agg_ptr.as<int>(),
                                                     C.agg_cells.as<int>(), F.t.as<float>(),
                                                     C.b.as<float>(), na);
    k += 2;
  }
  {
    MgLevel& C = *c->mg[L - 1];
    mg::k_mg_coarse_solve<<<1, mg::kCoarseBlock, 0, s>>>(C.n, c->mg_ainv.as<float>(),
                                                         C.b.as<float>(), C.y.as<float>(), na);
    k += 1;
  }
  for (int l = L - 2; l >= 0; --l) {
    MgLevel& F = *c->mg[l];
    MgLevel& C = *c->mg[l + 1];
    mg::k_mg_prolong<<<grid_for(c, F.n), B, 0, s>>>(F.n, C.agg_of.as<int>(), a, C.y.as<float>(),
                                                    F.x.as<float>(), na);
    with_chunk(c->row_chunk, [&](auto ch) {
      mg::k_mg_post<float, decltype(ch)::value><<<grid_for(c, F.n), B, 0, s>>>(
          F.n, F.rows(), F.dinv.as<float>(), w, F.b.as<float>(), F.x.as<float>(), F.y.as<float>(),
          na);
    });
    k += 2;
  }
  return k;
}

// z = one symmetric V-cycle applied to r (FP32, level 0 = the context's
// matrix).  Level 0 is smoothed by the network's operator (q, gE) for
// mode 1, by Jacobi with the network's per-cell weights q^2 for mode 2 and
// by damped Jacobi for mode 0.  x0 and t0 hold, afterwards, the level-0
// iterate before post-smoothing and its residual.  Returns the number of
// kernels launched.
template <typename TZ>
int mg_vcycle(solv_gpu_ctx* c, const float* r, TZ* z, int mode, const float* q, const float* ge,
              float* x0, float* t0, const int* na) {
  const bool net = mode == 1;
  cudaStream_t s = c->stream;
  const int B = c->block;
  const float w = (float)c->mg_omega, a = (float)c->mg_alpha;
  const int N = c->N;
  Rows<float> R0 = rows<float>(c);
  const float* d0 = mode == 2 ? c->mg_dq.as<float>() : c->mg_dinv0.as<float>();
  MgLevel& L1 = *c->mg[0];
  int k = 0;
  const int ch = c->row_chunk;
  if (net) {
    mg::k_mg_net<false, float><<<grid_resident(c, N), B, 0, s>>>(N, R0, ge, q, w, r, nullptr, x0, na);
    with_chunk(ch, [&](auto cc) {
      mg::k_mg_resid<decltype(cc)::value><<<grid_resident(c, N), B, 0, s>>>(N, R0, r, x0, t0, na);
    });
    k += 2;
  } else {
    with_chunk(ch, [&](auto cc) {
      mg::k_mg_pre<decltype(cc)::value><<<grid_resident(c, N), B, 0, s>>>(N, R0, d0, w, r, x0,
                                                                          t0, na);
    });
    k += 1;
  }
  mg::k_mg_restrict<<<grid_for(c, L1.n), B, 0, s>>>(L1.n, L1.agg_ptr.as<int>(),
                                                    L1.agg_cells.as<int>(), t0, L1.b.as<float>(),
                                                    na);
  k += 1 + mg_coarse_cycle(c, na);
  mg::k_mg_prolong<<<grid_resident(c, N), B, 0, s>>>(N, L1.agg_of.as<int>(), a, L1.y.as<float>(), x0,
                                                na);
  k += 1;
  if (net) {
    with_chunk(ch, [&](auto cc) {
      mg::k_mg_resid<decltype(cc)::value><<<grid_resident(c, N), B, 0, s>>>(N, R0, r, x0, t0, na);
    });
    mg::k_mg_net<true, TZ><<<grid_resident(c, N), B, 0, s>>>(N, R0, ge, q, w, t0, x0, z, na);
    k += 2;
  } else {
    with_chunk(ch, [&](auto cc) {
      mg::k_mg_post<TZ, decltype(cc)::value><<<grid_resident(c, N), B, 0, s>>>(N, R0, d0, w, r,
                                                                               x0, z, na);
    });
    k += 1;
  }
  return k;
}

// The solve uses the hierarchy (built, and not switched off).
bool mg_on(const solv_gpu_ctx* c) { return c->mg_max_levels > 0 && !c->mg.empty(); }

// A smoother must damp: with lambda_max(w K A) >= 2 some error modes grow
// under it and the V-cycle stops being a good preconditioner.  The network
// has no such bound built in -- a right-hand side far from its training
// data (a localised mass imbalance, say) can drive its per-cell scales up
// -- so every solve estimates lambda_max(w K A) by power iteration on the
// device and, above kSmoothMax, scales q = s D^-1/2 (the operator's only
// per-cell factor, K scaling with q^2) so that the bound holds.  The
// estimate is inflated by 5% (power iteration approaches lambda_max from
// below).  Before that the per-cell scales are held at or above
// mg_scale_min (default 0.5, a quarter of the Jacobi weight): a network that
// drives some s_i towards zero leaves those cells unsmoothed, which no bound
// on lambda_max sees.
// Returns the factor applied to K (1 when none was needed).
constexpr double kSmoothMax = 1.9;
constexpr int kPowerIters = 8;

int mg_bound_smoother(solv_gpu_ctx* c, double* applied) {
  *applied = 1.0;
  cudaStream_t s = c->stream;
  const int N = c->N;
  const int G = grid_for(c, N), B = c->block;
  Rows<float> R0 = rows<float>(c);
  float* v = c->mg_t0.as<float>();
  float* y = c->mg_x0.as<float>();
  CUDA_TRY(c, c->g_jsum.ensure(3 * sizeof(double)));
  double* acc = c->g_jsum.as<double>();
  mg::k_mg_floor<<<G, B, 0, s>>>(N, c->mg_scale_min, c->g_rsd.as<float>(), c->g_q.as<float>());
  mg::k_mg_hashfill<<<G, B, 0, s>>>(N, v);
  c->launches += 2;
  double prev = 0.0, lam = 0.0, h = 0.0;
  for (int it = 0; it <= kPowerIters; ++it) {
    CUDA_TRY(c, cudaMemsetAsync(acc, 0, sizeof(double), s));
    mg::k_mg_norm2<<<std::min(G, 1184), 256, 0, s>>>(N, v, acc);
    CUDA_TRY(c, cudaMemcpyAsync(&h, acc, sizeof(double), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(c, cudaStreamSynchronize(s));
    const double nrm = std::sqrt(h);
    if (!(nrm > 0.0) || !std::isfinite(nrm)) break;
    if (it > 0) lam = nrm / prev;  // |w K A v| / |v| for the previous, unit v
    if (it == kPowerIters) break;
    mg::k_mg_scale<<<G, B, 0, s>>>(N, (float)(1.0 / nrm), v);
    prev = 1.0;
    sg::k_spmv<float, 1><<<G, B, 0, s>>>(N, R0, v, y);  // y = A v
    mg::k_mg_net<false, float><<<G, B, 0, s>>>(N, R0, c->g_ge.as<float>(), c->g_q.as<float>(),
                                                (float)c->mg_omega, y, nullptr, v, nullptr);
    c->launches += 4;
  }
  CUDA_TRY(c, cudaGetLastError());
  lam *= 1.05;
  if (std::isfinite(lam) && lam > kSmoothMax) {
    const double f = kSmoothMax / lam;
    mg::k_mg_scale<<<G, B, 0, s>>>(N, (float)std::sqrt(f), c->g_q.as<float>());
    c->launches++;
    *applied = f;
  }
  CUDA_TRY(c, cudaGetLastError());
  return SOLV_GPU_OK;
}

// Kernels in one V-cycle (launch statistics of graph replays).
int mg_kernels(const solv_gpu_ctx* c) {
  const int L = (int)c->mg.size();
  const int fine = c->mg_smoother == 1 ? 5 : 3;  // smoothing, residual, prolongation
  return fine + 1 + 2 * (L - 1) + 1 + 2 * (L - 1);
}

// ---- building blocks -----------------------------------------------------------
template <int V>
void launch_res(solv_gpu_ctx* c, const double* phi, double* r, int not_r0) {
  sg::k_res<V><<<c->seg.total_blk, c->block, 0, c->stream>>>(
      rows<double>(c), segmap(c), phi, r, not_r0, c->part.as<double>(), c->l1.as<double>());
  c->launches++;
}

int run_res(solv_gpu_ctx* c, int V, const double* phi, double* r, int not_r0) {
  switch (V) {
    case 1: launch_res<1>(c, phi, r, not_r0); break;
    case 2: launch_res<2>(c, phi, r, not_r0); break;
    case 3: launch_res<3>(c, phi, r, not_r0); break;
    case 4: launch_res<4>(c, phi, r, not_r0); break;
    default: return set_err(c, SOLV_GPU_BAD_INPUT, "n_vc must be 1..4");
  }
  CUDA_TRY(c, cudaGetLastError());
  return SOLV_GPU_OK;
}

// Cooperative launch of a sync-free recurrence (kernels.cuh): every block
// resident at once, at most one warp per 32-cell slice.
template <typename... KArgs, typename... Args>
int coop_launch(solv_gpu_ctx* c, void (*kern)(KArgs...), Args... args) {
  auto it = c->coop_blocks.find((const void*)kern);
  int per_sm = 0;
  if (it != c->coop_blocks.end()) {
    per_sm = it->second;
  } else {
    CUDA_TRY(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, sg::kSweepThreads, 0));
    if (per_sm < 1) return set_err(c, SOLV_GPU_DEVICE_ERROR, "sweep kernel cannot be resident");
    c->coop_blocks[(const void*)kern] = per_sm;
  }
  const long long warps = ((long long)c->N + 31) / 32;
  const long long want = (warps + sg::kSweepThreads / 32 - 1) / (sg::kSweepThreads / 32);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)std::max(1LL, std::min<long long>(want, (long long)per_sm * c->n_sm)));
  cfg.blockDim = dim3(sg::kSweepThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = c->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  CUDA_TRY(c, cudaLaunchKernelEx(&cfg, kern, args...));
  c->launches++;
  return SOLV_GPU_OK;
}

sg::SweepCtl* sweep_ctl(solv_gpu_ctx* c) { return c->sweep_ctl.as<sg::SweepCtl>(); }

// A wait of a sweep ran out (SweepCtl::err): report it, clear the flag, and
// have the pending state of the sweep buffers rebuilt before the next use.
int sweep_check(solv_gpu_ctx* c) {
  sg::SweepCtl h{};
  CUDA_TRY(c, cudaMemcpyAsync(&h, c->sweep_ctl.p, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (!h.err) return SOLV_GPU_OK;
  CUDA_TRY(c, cudaMemsetAsync(c->sweep_ctl.p, 0, sizeof(sg::SweepCtl), c->stream));
  c->t_ready = c->tf_ready = false;
  return set_err(c, SOLV_GPU_TIMEOUT, "triangular sweep: a wait for a neighbour ran out");
}

// solv_precond: c, c_r in internal order (FP64).  DIC / DILU is one
// sync-free recurrence over the cells (c starts out pending).
int launch_precond(solv_gpu_ctx* c, int imat, double* cc, double* cr) {
  if (imat <= 0) {
    sg::k_precond_jacobi<<<grid_for(c, c->N), c->block, 0, c->stream>>>(c->N, c->diag.as<double>(),
                                                                         cc, cr);
    c->launches++;
    CUDA_TRY(c, cudaGetLastError());
    return SOLV_GPU_OK;
  }
  sg::k_fill_pending<double><<<grid_for(c, c->N), c->block, 0, c->stream>>>(c->N, cc);
  c->launches++;
  return coop_launch(c, sg::k_precond_sf, c->N, imat, rows<double>(c), (const int*)c->slot_src.as<int>(),
                     (const double*)c->fp.as<double>(), (const double*)c->fn.as<double>(), cc, cr,
                     sweep_ctl(c));
}

// x = M^-1 b  (solv_direct), internal order, V components: the forward
// sweep into the workspace t, the backward sweep from t into x (both
// sync-free recurrences, one cooperative launch each).
template <typename T>
T* sweep_t(solv_gpu_ctx* c) {
  if constexpr (std::is_same<T, double>::value) return c->w_t.as<double>();
  else return c->wf_t.as<float>();
}

template <typename T, int V>
int launch_direct(solv_gpu_ctx* c, int imat, const T* cc, const T* cr, T* x, const T* b,
                  const int* n_active) {
  if (imat <= 0) {
    sg::k_jacobi<T, V><<<grid_for(c, c->N), c->block, 0, c->stream>>>(c->N, cc, b, x);
    c->launches++;
    return SOLV_GPU_OK;
  }
  Rows<T> R = rows<T>(c);
  T* t = sweep_t<T>(c);
  int rc = coop_launch(c, sg::k_fwd_sf<T, V>, c->N, R, cc, b, t, x, sweep_ctl(c), n_active);
  if (rc) return rc;
  return coop_launch(c, sg::k_bwd_sf<T, V>, c->N, R, cc, cr, t, x, sweep_ctl(c), n_active);
}

// Workspace for V components in precision T.
template <typename T>
struct WS {
  T *phi, *r, *r0, *p, *q, *v, *z, *c, *cr, *t;
};

template <typename T>
int ensure_ws(solv_gpu_ctx* c, int V, WS<T>& w) {
  const size_t nv = (size_t)c->N * V * sizeof(T), n1 = (size_t)c->N * sizeof(T);
  bool f = std::is_same<T, float>::value;
  DevBuf* b[9];
  if (!f) {
    DevBuf* bd[9] = {&c->w_phi, &c->w_r, &c->w_r0, &c->w_p, &c->w_q, &c->w_v, &c->w_z, &c->w_c, &c->w_cr};
    std::copy(bd, bd + 9, b);
  } else {
    DevBuf* bf[9] = {&c->wf_phi, &c->wf_r, &c->wf_r0, &c->wf_p, &c->wf_q, &c->wf_v, &c->wf_z, &c->wf_c, &c->wf_cr};
    std::copy(bf, bf + 9, b);
  }
  for (int k = 0; k < 9; ++k) {
    void* old = b[k]->p;
    CUDA_TRY(c, b[k]->ensure(k < 7 ? nv : n1));
    if (old != b[k]->p) drop_graphs(c);
  }
  w.phi = b[0]->as<T>(); w.r = b[1]->as<T>(); w.r0 = b[2]->as<T>(); w.p = b[3]->as<T>();
  w.q = b[4]->as<T>(); w.v = b[5]->as<T>(); w.z = b[6]->as<T>(); w.c = b[7]->as<T>();
  w.cr = b[8]->as<T>();
  // the sweeps' t: all pending before every forward sweep
  DevBuf& tb = f ? c->wf_t : c->w_t;
  bool& ready = f ? c->tf_ready : c->t_ready;
  void* old = tb.p;
  CUDA_TRY(c, tb.ensure(nv));
  if (old != tb.p) {
    drop_graphs(c);
    ready = false;
  }
  if (!c->sweep_ctl.p) {
    CUDA_TRY(c, c->sweep_ctl.ensure(sizeof(sg::SweepCtl)));
    CUDA_TRY(c, cudaMemsetAsync(c->sweep_ctl.p, 0, sizeof(sg::SweepCtl), c->stream));
  }
  if (!ready) {
    sg::k_fill_pending<T><<<grid_for(c, (long long)c->N * V), c->block, 0, c->stream>>>(
        (long long)c->N * V, tb.as<T>());
    CUDA_TRY(c, cudaGetLastError());
    ready = true;
  }
  w.t = tb.as<T>();
  return SOLV_GPU_OK;
}

// q = A p with p.q (the CG product); FP32 products with the context's
// gather width.
template <typename T, int V>
void cg_spmv(solv_gpu_ctx* c, const SegMap& sm, WS<T>& w, double* part, Lane* lanes) {
  const int G = c->seg.total_blk, B = c->block;
  if constexpr (std::is_same<T, float>::value) {
    with_chunk(c->row_chunk, [&](auto ch) {
      sg::k_cg_spmv<T, V, decltype(ch)::value><<<G, B, 0, c->stream>>>(rows<T>(c), sm, w.p, w.q,
                                                                      part, lanes);
    });
  } else {
    sg::k_cg_spmv<T, V><<<G, B, 0, c->stream>>>(rows<T>(c), sm, w.p, w.q, part, lanes);
  }
}

// y = A z with its dots (BiCGSTAB, MODE as k_bi_spmv)
template <typename T, int V, int MODE>
void bi_spmv(solv_gpu_ctx* c, const SegMap& sm, const T* z, T* y, const T* wv, double* part,
             Lane* lanes) {
  const int G = c->seg.total_blk, B = c->block;
  if constexpr (std::is_same<T, float>::value) {
    with_chunk(c->row_chunk, [&](auto ch) {
      sg::k_bi_spmv<T, V, MODE, decltype(ch)::value><<<G, B, 0, c->stream>>>(rows<T>(c), sm, z, y,
                                                                            wv, part, lanes);
    });
  } else {
    sg::k_bi_spmv<T, V, MODE><<<G, B, 0, c->stream>>>(rows<T>(c), sm, z, y, wv, part, lanes);
  }
}

// One CG iteration (solv_cg.f90:37-84) on workspace w.  The FP32 inner
// iteration of the mixed-precision solve takes the flexible-CG step and
// direction formulas (FLEX in kernels.cuh): FP32 products lose the
// orthogonality the classic formulas rely on, and on a 256^3 pressure system
// the classic ones needed several times the FP64 iteration count.
template <typename T, int V>
int cg_iteration(solv_gpu_ctx* c, int imat, WS<T>& w) {
  constexpr bool FLEX = std::is_same<T, float>::value;
  SegMap sm = segmap(c);
  double* part = c->part.as<double>();
  Lane* lanes = c->lanes.as<Lane>();
  const int G = c->seg.total_blk, B = c->block;
  cudaStream_t st = c->stream;
  if (imat > 0) {
    if (int rc = launch_direct<T, V>(c, imat, w.c, w.cr, w.z, w.r, sm.n_active)) return rc;
    sg::k_cg_rz<T, V, false, FLEX><<<G, B, 0, st>>>(sm, w.c, w.r, w.z, part, lanes, w.q);
    sg::k_cg_p<T, V, false, FLEX><<<G, B, 0, st>>>(sm, w.c, w.r, w.z, w.p, lanes, part);
    cg_spmv<T, V>(c, sm, w, part, lanes);
    sg::k_cg_update<T, V, false, FLEX><<<G, B, 0, st>>>(sm, w.c, w.phi, w.r, w.p, w.q, part,
                                                        lanes);
    c->launches += 4;
  } else {
    sg::k_cg_p<T, V, true, FLEX><<<G, B, 0, st>>>(sm, w.c, w.r, w.z, w.p, lanes, part);
    cg_spmv<T, V>(c, sm, w, part, lanes);
    sg::k_cg_update<T, V, true, FLEX><<<G, B, 0, st>>>(sm, w.c, w.phi, w.r, w.p, w.q, part,
                                                       lanes);
    c->launches += 3;
  }
  return SOLV_GPU_OK;
}

// One BiCGSTAB iteration (solv_bicg.f90:42-118); rho/omeg of its head were
// produced by the previous k_bi_update (or k_bi_rho before the first).
template <typename T, int V>
int bicg_iteration(solv_gpu_ctx* c, int imat, WS<T>& w) {
  SegMap sm = segmap(c);
  double* part = c->part.as<double>();
  Lane* lanes = c->lanes.as<Lane>();
  const int G = c->seg.total_blk, B = c->block;
  cudaStream_t st = c->stream;
  // w.q holds u, w.v holds v
  if (imat > 0) {
    sg::k_bi_p<T, V, false><<<G, B, 0, st>>>(sm, w.c, w.r, w.p, w.q, w.z, lanes);
    if (int rc = launch_direct<T, V>(c, imat, w.c, w.cr, w.z, w.p, sm.n_active)) return rc;
  } else {
    sg::k_bi_p<T, V, true><<<G, B, 0, st>>>(sm, w.c, w.r, w.p, w.q, w.z, lanes);
  }
  bi_spmv<T, V, 0>(c, sm, w.z, w.q, w.r0, part, lanes);
  if (imat > 0) {
    sg::k_bi_half<T, V, false><<<G, B, 0, st>>>(sm, w.c, w.phi, w.r, w.z, w.q, lanes);
    if (int rc = launch_direct<T, V>(c, imat, w.c, w.cr, w.z, w.r, sm.n_active)) return rc;
  } else {
    sg::k_bi_half<T, V, true><<<G, B, 0, st>>>(sm, w.c, w.phi, w.r, w.z, w.q, lanes);
  }
  bi_spmv<T, V, 1>(c, sm, w.z, w.v, w.r, part, lanes);
  sg::k_bi_update<T, V><<<G, B, 0, st>>>(sm, w.phi, w.r, w.z, w.v, w.r0, part, lanes);
  c->launches += 5;
  return SOLV_GPU_OK;
}

// One flexible-CG iteration with the learned preconditioner (one system):
// z from one V-cycle of the aggregation hierarchy when one is built, else
// from the network's one-level operator.
template <typename T>
void fcg_iteration(solv_gpu_ctx* c, WS<T>& w) {
  SegMap sm = segmap(c);
  double* part = c->part.as<double>();
  Lane* lanes = c->lanes.as<Lane>();
  const int G = c->seg.total_blk, B = c->block;
  cudaStream_t st = c->stream;
  int nk = 1;
  if constexpr (std::is_same<T, float>::value) {
    if (mg_on(c))  // z = V-cycle(r)
      nk = mg_vcycle<T>(c, w.r, w.z, c->mg_smoother, c->g_q.as<float>(),
                        c->g_ge.as<float>(), c->mg_x0.as<float>(), c->mg_t0.as<float>(),
                        sm.n_active);
  }
  if (!mg_on(c))
    gnn::k_gnn_apply<T><<<grid_for(c, c->N), B, 0, st>>>(c->N, rows<float>(c),
                                                          c->g_ge.as<float>(), c->g_q.as<float>(),
                                                          w.r, w.z, sm.n_active);  // z = M^-1 r
  c->launches += nk - 1;
  sg::k_fcg_beta<T><<<G, B, 0, st>>>(sm, w.z, w.q, part, lanes);            // beta
  sg::k_cg_p<T, 1, false><<<G, B, 0, st>>>(sm, w.c, w.r, w.z, w.p, lanes);   // p = z + beta p
  with_chunk(c->row_chunk, [&](auto ch) {
    sg::k_fcg_spmv<T, decltype(ch)::value><<<G, B, 0, st>>>(rows<T>(c), sm, w.p, w.q, w.r, part,
                                                            lanes);
  });
  sg::k_fcg_update<T><<<G, B, 0, st>>>(sm, w.phi, w.r, w.p, w.q, part, lanes);
  c->launches += 5;
}

// The preconditioner part of a graph's key: the recurrence (imat) for CG
// and BiCGSTAB, the V-cycle's smoother for the learned FCG (a solve may
// switch it, and both graphs stay cached).
int graph_imat_key(const solv_gpu_ctx* c, int solver, int imat) {
  if (solver == 2) return 10 + c->mg_smoother;
  return imat > 0 ? imat : 0;
}

// A WHILE graph of one Krylov iteration (body) and the loop control: a
// launch runs iterations until every lane has stopped or the budget in
// c->loop_budget is spent, with no host round trip in between.  Returns the
// CUDA error of building it (conditional nodes unsupported, or a node the
// body graph cannot hold); rc carries body()'s own status.
template <typename Body>
cudaError_t build_while_graph(solv_gpu_ctx* c, Body&& body, int& rc, cudaGraphExec_t& exec) {
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaGraphCreate(&g, 0);
  if (e != cudaSuccess) return e;
  cudaGraphConditionalHandle h;
  e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
  if (e == cudaSuccess) {
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    e = cudaGraphAddNode(&node, g, nullptr, 0, &p);
    if (e == cudaSuccess) {
      cudaGraph_t bg = p.conditional.phGraph_out[0];
      e = cudaStreamBeginCaptureToGraph(c->stream, bg, nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        rc = body();
        if (!rc)
          sg::k_loop_ctl<<<1, 32, 0, c->stream>>>(h, c->n_active.as<int>(),
                                                  c->loop_budget.as<int>());
        cudaGraph_t out = nullptr;
        const cudaError_t e2 = cudaStreamEndCapture(c->stream, &out);
        if (e == cudaSuccess) e = e2;
      }
      if (e == cudaSuccess && !rc) e = cudaGraphInstantiate(&exec, g, 0);
    }
  }
  cudaGraphDestroy(g);
  return e;
}

// Run Krylov iterations until every lane stops (device counter): one launch
// of a WHILE graph where conditional nodes are available, else
// `graph_iters` iterations per CUDA-graph launch.
template <typename T, int V>
int iterate(solv_gpu_ctx* c, int solver, int imat, int n_iter, WS<T>& w, int& graph_launches) {
  const int K = c->graph_iters;
  auto body = [&]() -> int {
    if (solver == 0) return cg_iteration<T, V>(c, imat, w);
    if (solver == 1) return bicg_iteration<T, V>(c, imat, w);
    if constexpr (V == 1) fcg_iteration<T>(c, w);
    return SOLV_GPU_OK;
  };
  cudaGraphExec_t exec = nullptr;
  bool loop = false;  // exec is a WHILE graph: one launch runs until the lanes stop
  // WHILE graphs where lanes stop inside a graph for reliable updates (the
  // learned FCG), fixed ones elsewhere (a WHILE pass costs ~3 us)
  const bool want_loop = c->graph_loop == 1 || (c->graph_loop == 2 && solver == 2);
  if (K > 0 && want_loop && c->cond_graphs) {
    auto key = std::make_tuple(solver, graph_imat_key(c, solver, imat), V,
                               (int)std::is_same<T, float>::value, 1);
    auto it = c->graphs.find(key);
    if (it != c->graphs.end()) {
      exec = it->second;  // null: this body cannot be a WHILE graph
      loop = exec != nullptr;
    } else {
      CUDA_TRY(c, c->loop_budget.ensure(sizeof(int)));
      int l0 = c->launches;
      int rc = SOLV_GPU_OK;
      cudaError_t e = build_while_graph(c, body, rc, exec);
      c->launches = l0;
      if (rc) return rc;
      if (e == cudaSuccess) {
        c->graphs[key] = exec;
        loop = true;
      } else {  // not as a WHILE graph: K iterations per launch instead
        cudaGetLastError();
        if (e == cudaErrorNotSupported || e == cudaErrorCallRequiresNewerDriver)
          c->cond_graphs = false;  // no conditional nodes at all
        else
          c->graphs[key] = nullptr;  // this body only
        exec = nullptr;
      }
    }
  }
  if (K > 0 && !loop) {
    auto key = std::make_tuple(solver, graph_imat_key(c, solver, imat), V,
                               (int)std::is_same<T, float>::value, 0);
    auto it = c->graphs.find(key);
    if (it != c->graphs.end()) {
      exec = it->second;
    } else {
      cudaGraph_t g;
      CUDA_TRY(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      int l0 = c->launches;
      int rc = SOLV_GPU_OK;
      for (int k = 0; k < K && !rc; ++k) rc = body();
      cudaError_t e = cudaStreamEndCapture(c->stream, &g);
      c->launches = l0;
      if (rc) {
        if (e == cudaSuccess) cudaGraphDestroy(g);
        return rc;
      }
      CUDA_TRY(c, e);
      e = cudaGraphInstantiate(&exec, g, 0);
      cudaGraphDestroy(g);
      CUDA_TRY(c, e);
      c->graphs[key] = exec;
    }
  }
  int done = 0;
  int per_launch_kernels = 0;
  {
    // kernels per iteration (for the launch count statistics)
    int l0 = c->launches;
    // count by dry accounting: replicate the arithmetic of body()
    int sweep = imat > 0 ? 2 : 1;  // forward + backward recurrence, or Jacobi
    if (solver == 0) per_launch_kernels = imat > 0 ? sweep + 4 : 3;
    else if (solver == 1) per_launch_kernels = imat > 0 ? 2 * sweep + 5 : 5;
    else per_launch_kernels = 4 + (mg_on(c) ? mg_kernels(c) : 1);
    c->launches = l0;
  }
  while (done < n_iter) {
    if (loop) {  // up to n_iter - done iterations in one launch
      const int b = n_iter - done;
      c->h_n_active[1] = b;
      CUDA_TRY(c, cudaMemcpyAsync(c->loop_budget.p, &c->h_n_active[1], sizeof(int),
                                  cudaMemcpyHostToDevice, c->stream));
      CUDA_TRY(c, cudaGraphLaunch(exec, c->stream));
      CUDA_TRY(c, cudaMemcpyAsync(&c->h_n_active[1], c->loop_budget.p, sizeof(int),
                                  cudaMemcpyDeviceToHost, c->stream));
      graph_launches++;
    } else if (exec) {
      CUDA_TRY(c, cudaGraphLaunch(exec, c->stream));
      graph_launches++;
      c->launches += K * per_launch_kernels;
      done += K;
    } else {
      if (int rc = body()) return rc;
      done += 1;
    }
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, cudaMemcpyAsync(c->h_n_active, c->n_active.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    if (loop) {
      const int ran = std::max(1, n_iter - done - c->h_n_active[1]);
      c->launches += ran * (per_launch_kernels + 1);
      done += ran;
    }
    if (*c->h_n_active <= 0) break;
  }
  return SOLV_GPU_OK;
}

// Full FP64 solve (solver 0 = CG, 1 = BiCGSTAB) on device buffers in the
// caller layouts.
template <int V>
int solve_fp64(solv_gpu_ctx* c, int solver, int imat, double reduc, int n_iter,
               double* phi_dev, double* res0_dev, double* res0_n, int not_r0,
               solv_gpu_stats* st, int* out_iters, double* out_ratio) {
  WS<double> w;
  int rc = ensure_ws<double>(c, V, w);
  if (rc) return rc;
  const int N = c->N;
  cudaStream_t s = c->stream;
  const int* o2n = c->old_of_new.as<int>();
  sg::k_phi_in<double><<<grid_for(c, N), c->block, 0, s>>>(N, V, o2n, phi_dev, w.phi);
  sg::k_col_in<<<grid_for(c, N), c->block, 0, s>>>(N, V, o2n, res0_dev, w.r0);
  c->launches += 2;
  const int nl = c->n_seg * V;
  rc = run_res(c, V, w.phi, w.r0, not_r0);  // solv_res: r0 = b - A phi, res0_n
  if (rc) return rc;
  sg::k_set_res0n<<<1, 256, 0, s>>>(c->lanes.as<Lane>(), nl, c->l1.as<double>());
  // res0 out = initial residual (solv_cg.f90:20)
  sg::k_col_out<<<grid_for(c, N), c->block, 0, s>>>(N, V, o2n, w.r0, res0_dev);
  c->launches++;
  std::vector<Lane> hl(nl);
  CUDA_TRY(c, cudaMemcpyAsync(res0_n, c->l1.p, nl * sizeof(double), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(c, cudaStreamSynchronize(s));
  double mx = -HUGE_VAL;
  for (int l = 0; l < nl; ++l) mx = std::max(mx, res0_n[l]);
  if (st) st->n_vc = V;
  if (mx < sg::kSmall) {  // solv_cg.f90:21 early return
    if (st) st->status = SOLV_GPU_ZERO_RHS;
    if (out_iters) std::fill(out_iters, out_iters + nl, 0);
    if (out_ratio) std::fill(out_ratio, out_ratio + nl, 0.0);
    return SOLV_GPU_OK;
  }
  if ((rc = launch_precond(c, imat, w.c, w.cr))) return rc;  // solv_precond
  CUDA_TRY(c, cudaMemcpyAsync(w.r, w.r0, (size_t)N * V * sizeof(double), cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(c, cudaMemsetAsync(w.p, 0, (size_t)N * V * sizeof(double), s));
  CUDA_TRY(c, cudaMemsetAsync(w.q, 0, (size_t)N * V * sizeof(double), s));
  CUDA_TRY(c, cudaMemsetAsync(w.v, 0, (size_t)N * V * sizeof(double), s));
  CUDA_TRY(c, cudaMemsetAsync(w.z, 0, (size_t)N * V * sizeof(double), s));
  {
    int na = nl;
    if (n_iter <= 0) na = 0;
    CUDA_TRY(c, cudaMemcpyAsync(c->n_active.p, &na, sizeof(int), cudaMemcpyHostToDevice, s));
  }
  sg::k_lane_init<<<(nl + 255) / 256, 256, 0, s>>>(c->lanes.as<Lane>(), nl, n_iter, reduc,
                                                   c->n_active.as<int>());
  SegMap sm = segmap(c);
  const bool fused = c->persistent && solver == 0 && imat <= 0 && V == 1;
  if (solver == 0) {
    if (imat <= 0 && !fused) {
      sg::k_cg_rz<double, V, true><<<c->seg.total_blk, c->block, 0, s>>>(
          sm, w.c, w.r, w.z, c->part.as<double>(), c->lanes.as<Lane>());
      c->launches++;
    }
  } else {
    sg::k_bi_rho<double, V><<<c->seg.total_blk, c->block, 0, s>>>(
        sm, w.r, w.r0, c->part.as<double>(), c->lanes.as<Lane>());
    c->launches++;
  }
  c->launches += 2;
  CUDA_TRY(c, cudaGetLastError());
  int gl = 0;
  if (fused) {  // the whole loop in one launch: one cluster per system
    // systems of at most 16 x 2048 cells run with their vectors in the
    // cluster's registers and shared memory (k_pcg_cluster_res), larger
    // ones from global memory (k_pcg_cluster); 16 blocks per cluster where
    // all the systems' clusters fit at once, else the portable 8
    int maxn = 0;
    for (size_t k = 0; k < c->seg_c0_caller.size(); ++k)
      maxn = std::max(maxn, c->seg_c1_caller[k] - c->seg_c0_caller[k]);
    using PcgKernel = void (*)(Rows<double>, const int*, const int*, const double*, double*,
                               double*, double*, double*, Lane*, int*);
    auto clusters16 = [&](PcgKernel kern) {
      auto it = c->pcg_max16.find((const void*)kern);
      if (it != c->pcg_max16.end()) return it->second;
      int n16 = 0;
      if (cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
          cudaSuccess) {
        cudaLaunchConfig_t qc = {};
        qc.gridDim = dim3(sg::kPcgClusterMax);
        qc.blockDim = dim3(sg::kPcgThreads);
        cudaLaunchAttribute qa[1];
        qa[0].id = cudaLaunchAttributeClusterDimension;
        qa[0].val.clusterDim.x = sg::kPcgClusterMax;
        qa[0].val.clusterDim.y = 1;
        qa[0].val.clusterDim.z = 1;
        qc.attrs = qa;
        qc.numAttrs = 1;
        if (cudaOccupancyMaxActiveClusters(&n16, kern, &qc) != cudaSuccess) n16 = 0;
      }
      cudaGetLastError();  // a refused query leaves the portable size
      c->pcg_max16[(const void*)kern] = n16;
      return n16;
    };
    // the resident form reads a neighbour's p from the block that owns it:
    // fast where most neighbours are in the reader's own block (RCM-like
    // orders), slower than L2 where a warp's neighbours scatter over the
    // cluster (a permuted order), so it runs only on mostly local structures
    auto local_share = [&](int logb) -> double {
      auto it = c->pcg_local.find(logb);
      if (it != c->pcg_local.end()) return it->second;
      unsigned long long h[2] = {0, 0};
      DevBuf cnt;
      if (cnt.ensure(2 * sizeof(unsigned long long)) != cudaSuccess) return 0.0;
      cudaMemsetAsync(cnt.p, 0, 2 * sizeof(unsigned long long), s);
      sg::k_block_locality<<<grid_for(c, N), c->block, 0, s>>>(
          N, rows<double>(c), sm.seg_c0, sm.seg_c1, c->n_seg, logb,
          cnt.as<unsigned long long>());
      cudaMemcpyAsync(h, cnt.p, sizeof(h), cudaMemcpyDeviceToHost, s);
      if (cudaStreamSynchronize(s) != cudaSuccess) return 0.0;
      const double f = h[0] ? (double)h[1] / (double)h[0] : 1.0;
      c->pcg_local[logb] = f;
      return f;
    };
    PcgKernel kern = sg::k_pcg_cluster;
    int cs = sg::kPcgCluster;
    const PcgKernel res[2] = {sg::k_pcg_cluster_res<1>, sg::k_pcg_cluster_res<2>};
    for (int rpt = 1; rpt <= 2 && kern == sg::k_pcg_cluster; ++rpt) {
      const int cap = sg::kPcgThreads * rpt;
      if (maxn > sg::kPcgClusterMax * cap || local_share(rpt == 1 ? 10 : 11) < 0.5) continue;
      if (c->n_seg <= clusters16(res[rpt - 1]) && maxn <= sg::kPcgClusterMax * cap) {
        kern = res[rpt - 1];
        cs = sg::kPcgClusterMax;
      } else if (maxn <= sg::kPcgCluster * cap) {
        kern = res[rpt - 1];
        cs = sg::kPcgCluster;
      }
    }
    if (kern == sg::k_pcg_cluster && c->n_seg <= clusters16(kern)) cs = sg::kPcgClusterMax;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(c->n_seg * cs));
    cfg.blockDim = dim3(sg::kPcgThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CUDA_TRY(c, cudaLaunchKernelEx(&cfg, kern, rows<double>(c), sm.seg_c0, sm.seg_c1,
                                   (const double*)w.c, w.phi, w.r, w.p, w.q, c->lanes.as<Lane>(),
                                   c->n_active.as<int>()));
    c->launches++;
  } else {
    rc = iterate<double, V>(c, solver, imat, n_iter, w, gl);
    if (rc) return rc;
  }
  sg::k_phi_out<double><<<grid_for(c, N), c->block, 0, s>>>(N, V, o2n, w.phi, phi_dev);
  c->launches++;
  CUDA_TRY(c, cudaMemcpyAsync(hl.data(), c->lanes.p, nl * sizeof(Lane), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(c, cudaStreamSynchronize(s));
  int status = SOLV_GPU_OK;
  for (int l = 0; l < nl; ++l) {
    if (hl[l].status == sg::kLaneNaN) status = SOLV_GPU_NAN;
    else if (hl[l].status != sg::kLaneConverged && status == SOLV_GPU_OK) status = SOLV_GPU_MAXITER;
    if (out_iters) out_iters[l] = hl[l].iter;
    if (out_ratio) out_ratio[l] = hl[l].ratio;
  }
  if (st) {
    for (int v = 0; v < V && v < nl; ++v) {
      st->iters[v] = hl[v].iter;
      st->ratio[v] = hl[v].ratio;
    }
    st->status = status;
    st->graph_launches += gl;
  }
  return status;
}

// Mixed precision: FP32 inner Krylov solves of A d = r inside an FP64
// iterative-refinement loop.  FP64 stays on the device for the outer
// residual r = b - A x (k_res, bit-exact with the oracle's solv_res), the
// inner products (every reduction accumulates in FP64) and the solution
// accumulation x += d.  The stopping rule is the reference's, applied to
// the true FP64 residual: |b - A x|_1 / |r0|_1 < reduc.
template <int V>
int solve_mixed(solv_gpu_ctx* c, int solver, int imat, double reduc, int n_iter,
                double* phi_dev, double* res0_dev, double* res0_n, int not_r0,
                solv_gpu_stats* st, int* out_iters, double* out_ratio) {
  WS<double> w;
  WS<float> f;
  int rc = ensure_ws<double>(c, V, w);
  if (rc) return rc;
  if ((rc = ensure_ws<float>(c, V, f))) return rc;
  {
    void* old = c->valf.p;
    if ((rc = ensure_f32_matrix(c))) return rc;
    if (old != c->valf.p) drop_graphs(c);
  }
  const int N = c->N;
  const int nl = c->n_seg * V;
  const long long NV = (long long)N * V;
  cudaStream_t s = c->stream;
  const int* o2n = c->old_of_new.as<int>();
  CUDA_TRY(c, c->mp_mask.ensure(nl * sizeof(int)));
  double* b = w.q;  // the right-hand side, kept for the outer residuals
  sg::k_phi_in<double><<<grid_for(c, N), c->block, 0, s>>>(N, V, o2n, phi_dev, w.phi);
  sg::k_col_in<<<grid_for(c, N), c->block, 0, s>>>(N, V, o2n, res0_dev, b);
  CUDA_TRY(c, cudaMemcpyAsync(w.r0, b, NV * sizeof(double), cudaMemcpyDeviceToDevice, s));
  c->launches += 2;
  // not_r0: b is already the residual of the incoming phi, so refine a
  // correction from zero and add the incoming phi back at the end
  if (not_r0) {
    CUDA_TRY(c, cudaMemcpyAsync(w.v, w.phi, NV * sizeof(double), cudaMemcpyDeviceToDevice, s));
    CUDA_TRY(c, cudaMemsetAsync(w.phi, 0, NV * sizeof(double), s));
  }
  if ((rc = run_res(c, V, w.phi, w.r0, not_r0))) return rc;
  sg::k_col_out<<<grid_for(c, N), c->block, 0, s>>>(N, V, o2n, w.r0, res0_dev);
  c->launches++;
  std::vector<double> l1(nl);
  CUDA_TRY(c, cudaMemcpyAsync(l1.data(), c->l1.p, nl * sizeof(double), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(c, cudaStreamSynchronize(s));
  double mx = -HUGE_VAL;
  for (int l = 0; l < nl; ++l) {
    res0_n[l] = l1[l];
    mx = std::max(mx, l1[l]);
  }
  if (st) st->n_vc = V;
  if (mx < sg::kSmall) {
    if (st) st->status = SOLV_GPU_ZERO_RHS;
    if (out_iters) std::fill(out_iters, out_iters + nl, 0);
    if (out_ratio) std::fill(out_ratio, out_ratio + nl, 0.0);
    return SOLV_GPU_OK;
  }
  // preconditioner in FP64 (solv_precond), rounded to FP32 for the sweeps
  if ((rc = launch_precond(c, imat, w.c, w.cr))) return rc;
  sg::k_convert<double, float><<<grid_for(c, N), c->block, 0, s>>>(N, w.c, f.c);
  sg::k_convert<double, float><<<grid_for(c, N), c->block, 0, s>>>(N, w.cr, f.cr);
  c->launches += 2;

  std::vector<int> iters(nl, 0), status_v(nl), stalls(nl, 0), mask(nl);
  std::vector<double> ratio(nl), prev(nl);
  std::vector<char> active(nl);
  for (int l = 0; l < nl; ++l) {
    ratio[l] = l1[l] / (res0_n[l] + sg::kSmall);
    prev[l] = ratio[l];
    active[l] = !(ratio[l] < reduc) && n_iter > 0;
    status_v[l] = active[l] ? sg::kLaneRunning : (n_iter > 0 ? sg::kLaneConverged : sg::kLaneMaxIter);
  }
  const double* rcur = w.r0;  // current FP64 residual
  int refinements = 0, gl_total = 0;
  bool gnn_ok = true;
  c->fallbacks = 0;
  std::vector<Lane> hl(nl);
  for (int k = 0; k < c->max_refine; ++k) {
    int na = 0, cap = 0;
    for (int l = 0; l < nl; ++l) {
      Lane L{};
      L.s = sg::kLarge; L.alpha = 1.0; L.beta0 = 1.0; L.gam = 1.0;
      L.res0_n = l1[l];
      // do not over-solve the last sweep: the inner drop needed to reach reduc
      double need = 0.3 * reduc * (res0_n[l] + sg::kSmall) / (l1[l] + sg::kSmall);
      L.reduc = std::min(0.5, std::max(c->inner_reduc, need));
      // an FP32 sweep that cannot reach its drop (rounding floor) must not
      // run to the outer cap: bound each sweep, the outer loop decides
      L.n_iter = std::min(n_iter - iters[l], c->inner_max_iter);
      L.active = active[l] && L.n_iter > 0;
      L.status = sg::kLaneRunning;
      mask[l] = L.active;
      if (L.active) { ++na; cap = std::max(cap, L.n_iter); }
      hl[l] = L;
    }
    if (na == 0) break;
    ++refinements;
    CUDA_TRY(c, cudaMemcpyAsync(c->lanes.p, hl.data(), nl * sizeof(Lane), cudaMemcpyHostToDevice, s));
    CUDA_TRY(c, cudaMemcpyAsync(c->mp_mask.p, mask.data(), nl * sizeof(int), cudaMemcpyHostToDevice, s));
    CUDA_TRY(c, cudaMemcpyAsync(c->n_active.p, &na, sizeof(int), cudaMemcpyHostToDevice, s));
    sg::k_mp_start<V><<<grid_for(c, NV), c->block, 0, s>>>(NV, rcur, f.r, f.r0, f.phi);
    CUDA_TRY(c, cudaMemsetAsync(f.p, 0, NV * sizeof(float), s));
    CUDA_TRY(c, cudaMemsetAsync(f.q, 0, NV * sizeof(float), s));
    CUDA_TRY(c, cudaMemsetAsync(f.v, 0, NV * sizeof(float), s));
    CUDA_TRY(c, cudaMemsetAsync(f.z, 0, NV * sizeof(float), s));
    SegMap sm = segmap(c);
    // the learned preconditioner runs until it fails once; then plain PCG
    const int inner = (solver == 2 && !gnn_ok) ? 0 : solver;
    if (inner == 0) {
      if (imat <= 0) {
        sg::k_cg_rz<float, V, true><<<c->seg.total_blk, c->block, 0, s>>>(
            sm, f.c, f.r, f.z, c->part.as<double>(), c->lanes.as<Lane>());
        c->launches++;
      }
    } else if (inner == 1) {
      sg::k_bi_rho<float, V><<<c->seg.total_blk, c->block, 0, s>>>(
          sm, f.r, f.r0, c->part.as<double>(), c->lanes.as<Lane>());
      c->launches++;
    } else {
      if ((rc = gnn_prepare(c))) return rc;
      sg::k_fcg_scale<float><<<c->seg.total_blk, c->block, 0, s>>>(
          sm, f.r, c->g_rsd.as<float>(), c->part.as<double>(), c->lanes.as<Lane>());
      gnn_build<float>(c, f.r);
      c->launches++;
    }
    c->launches++;
    CUDA_TRY(c, cudaGetLastError());
    int gl = 0;
    if ((rc = iterate<float, V>(c, inner, imat, cap, f, gl))) return rc;
    gl_total += gl;
    CUDA_TRY(c, cudaMemcpyAsync(hl.data(), c->lanes.p, nl * sizeof(Lane), cudaMemcpyDeviceToHost, s));
    // x += d in FP64, then the true residual r = b - A x in FP64
    sg::k_mp_accum<V><<<c->seg.total_blk, c->block, 0, s>>>(sm, c->mp_mask.as<int>(), w.phi, f.phi);
    CUDA_TRY(c, cudaMemcpyAsync(w.r, b, NV * sizeof(double), cudaMemcpyDeviceToDevice, s));
    if ((rc = run_res(c, V, w.phi, w.r, 0))) return rc;
    c->launches += 2;
    rcur = w.r;
    CUDA_TRY(c, cudaMemcpyAsync(l1.data(), c->l1.p, nl * sizeof(double), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(c, cudaStreamSynchronize(s));
    for (int l = 0; l < nl; ++l) {
      if (!mask[l]) continue;
      iters[l] += hl[l].iter;
      ratio[l] = l1[l] / (res0_n[l] + sg::kSmall);
      if (!(ratio[l] == ratio[l]) || std::isinf(ratio[l]) || hl[l].status == sg::kLaneNaN) {
        active[l] = false;
        status_v[l] = sg::kLaneNaN;
      } else if (ratio[l] < reduc) {
        active[l] = false;
        status_v[l] = sg::kLaneConverged;
      } else if (iters[l] >= n_iter) {
        active[l] = false;
        status_v[l] = sg::kLaneMaxIter;
      } else if (inner == 2 && (hl[l].status == sg::kLaneStall || ratio[l] > 0.5 * prev[l])) {
        // the learned preconditioner stalled (or lost positive curvature):
        // plain PCG takes over from the current iterate
        gnn_ok = false;
        c->fallbacks++;
      } else {
        // a sweep that does not halve the residual twice running: FP32 has
        // reached its floor on this system
        stalls[l] = ratio[l] > 0.5 * prev[l] ? stalls[l] + 1 : 0;
        if (stalls[l] >= 2) {
          active[l] = false;
          status_v[l] = sg::kLaneMaxIter;
        }
      }
      prev[l] = ratio[l];
    }
  }
  for (int l = 0; l < nl; ++l)
    if (active[l]) status_v[l] = sg::kLaneMaxIter;  // refinement cap
  if (not_r0) {
    sg::k_add<<<grid_for(c, NV), c->block, 0, s>>>(NV, w.phi, w.v);
    c->launches++;
  }
  sg::k_phi_out<double><<<grid_for(c, N), c->block, 0, s>>>(N, V, o2n, w.phi, phi_dev);
  c->launches++;
  CUDA_TRY(c, cudaGetLastError());
  int status = SOLV_GPU_OK;
  for (int l = 0; l < nl; ++l) {
    if (status_v[l] == sg::kLaneNaN) status = SOLV_GPU_NAN;
    else if (status_v[l] != sg::kLaneConverged && status == SOLV_GPU_OK) status = SOLV_GPU_MAXITER;
    if (out_iters) out_iters[l] = iters[l];
    if (out_ratio) out_ratio[l] = ratio[l];
  }
  if (st) {
    for (int v = 0; v < V && v < nl; ++v) {
      st->iters[v] = iters[v];
      st->ratio[v] = ratio[v];
    }
    st->status = status;
    st->refinements = refinements;
    st->fallbacks = c->fallbacks;
    st->graph_launches += gl_total;
  }
  return status;
}

// Mixed-precision CG / FCG with reliable updates: the Krylov iteration runs
// in FP32 without restarts; whenever a lane's FP32 recursive residual has
// dropped by `reliable_delta` since the last update (or claims
// convergence), the FP32 correction is added to the FP64 solution, the
// FP64 residual b - A x replaces the FP32 one, and the search direction
// carries on.  Only the FP64 residual decides convergence.  A flexible-CG
// lane of the learned preconditioner stops itself at that drop
// (Lane::l1_stop, kLaneRefine), whatever the graph length: iterations past
// it would only push the FP32 recursive residual below what FP32 can
// represent of the true one.  Jacobi-CG lanes are checked between graph
// launches only: on a pinned Poisson system their slowest mode (the one the
// pin barely holds) converges late relative to the residual, and stopping
// each lane at the first 0.1 drop left it 1e-7 off at a 1e-10 residual.
template <int V>
int solve_mixed_reliable(solv_gpu_ctx* c, int solver, int imat, double reduc, int n_iter,
                         double* phi_dev, double* res0_dev, double* res0_n, int not_r0,
                         solv_gpu_stats* st, int* out_iters, double* out_ratio) {
  WS<double> w;
  WS<float> f;
  int rc = ensure_ws<double>(c, V, w);
  if (rc) return rc;
  if ((rc = ensure_ws<float>(c, V, f))) return rc;
  {
    void* old = c->valf.p;
    if ((rc = ensure_f32_matrix(c))) return rc;
    if (old != c->valf.p) drop_graphs(c);
  }
  const int N = c->N;
  const int nl = c->n_seg * V;
  const long long NV = (long long)N * V;
  cudaStream_t s = c->stream;
  const int* o2n = c->old_of_new.as<int>();
  CUDA_TRY(c, c->mp_mask.ensure(nl * sizeof(int)));
  double* b = w.q;
  sg::k_phi_in<double><<<grid_for(c, N), c->block, 0, s>>>(N, V, o2n, phi_dev, w.phi);
  sg::k_col_in<<<grid_for(c, N), c->block, 0, s>>>(N, V, o2n, res0_dev, b);
  CUDA_TRY(c, cudaMemcpyAsync(w.r0, b, NV * sizeof(double), cudaMemcpyDeviceToDevice, s));
  c->launches += 2;
  if (not_r0) {
    CUDA_TRY(c, cudaMemcpyAsync(w.v, w.phi, NV * sizeof(double), cudaMemcpyDeviceToDevice, s));
    CUDA_TRY(c, cudaMemsetAsync(w.phi, 0, NV * sizeof(double), s));
  }
  if ((rc = run_res(c, V, w.phi, w.r0, not_r0))) return rc;
  sg::k_col_out<<<grid_for(c, N), c->block, 0, s>>>(N, V, o2n, w.r0, res0_dev);
  c->launches++;
  std::vector<double> l1(nl);
  CUDA_TRY(c, cudaMemcpyAsync(l1.data(), c->l1.p, nl * sizeof(double), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(c, cudaStreamSynchronize(s));
  double mx = -HUGE_VAL;
  for (int l = 0; l < nl; ++l) {
    res0_n[l] = l1[l];
    mx = std::max(mx, l1[l]);
  }
  if (st) st->n_vc = V;
  if (mx < sg::kSmall) {
    if (st) st->status = SOLV_GPU_ZERO_RHS;
    if (out_iters) std::fill(out_iters, out_iters + nl, 0);
    if (out_ratio) std::fill(out_ratio, out_ratio + nl, 0.0);
    return SOLV_GPU_OK;
  }
  if ((rc = launch_precond(c, imat, w.c, w.cr))) return rc;
  sg::k_convert<double, float><<<grid_for(c, N), c->block, 0, s>>>(N, w.c, f.c);
  sg::k_convert<double, float><<<grid_for(c, N), c->block, 0, s>>>(N, w.cr, f.cr);
  sg::k_mp_start<V><<<grid_for(c, NV), c->block, 0, s>>>(NV, w.r0, f.r, f.r0, f.phi);
  CUDA_TRY(c, cudaMemsetAsync(f.p, 0, NV * sizeof(float), s));
  CUDA_TRY(c, cudaMemsetAsync(f.q, 0, NV * sizeof(float), s));
  CUDA_TRY(c, cudaMemsetAsync(f.z, 0, NV * sizeof(float), s));
  c->launches += 3;

  std::vector<Lane> hl(nl);
  std::vector<double> ratio(nl), l1_last(nl);
  std::vector<int> final_(nl, 0), status_v(nl, sg::kLaneRunning), stalls(nl, 0), mask(nl, 0);
  int na = 0;
  for (int l = 0; l < nl; ++l) {
    Lane L{};
    L.s = sg::kLarge; L.alpha = 1.0; L.beta0 = 1.0; L.gam = 1.0;
    L.res0_n = res0_n[l];
    L.l1 = l1[l];
    L.reduc = reduc;
    L.n_iter = n_iter;
    ratio[l] = l1[l] / (res0_n[l] + sg::kSmall);
    L.active = !(ratio[l] < reduc) && n_iter > 0;
    if (!L.active) {
      final_[l] = 1;
      status_v[l] = n_iter > 0 ? sg::kLaneConverged : sg::kLaneMaxIter;
    }
    L.status = sg::kLaneRunning;
    l1_last[l] = l1[l];
    // the learned FCG lane stops itself for the update (Jacobi CG lanes are
    // checked between graph launches: their near-null modes want the longer runs)
    L.l1_stop = solver == 2 ? c->fcg_reliable_delta * l1[l] : 0.0;
    na += L.active;
    hl[l] = L;
  }
  CUDA_TRY(c, cudaMemcpyAsync(c->lanes.p, hl.data(), nl * sizeof(Lane), cudaMemcpyHostToDevice, s));
  CUDA_TRY(c, cudaMemcpyAsync(c->n_active.p, &na, sizeof(int), cudaMemcpyHostToDevice, s));
  SegMap sm = segmap(c);
  const int G = c->seg.total_blk, B = c->block;
  if (solver == 2) {  // the learned preconditioner of this solve, from r0
    if (c->mg_max_levels > 0 && (rc = mg_setup(c))) return rc;  // may build no levels
    if (!mg_on(c) || c->mg_smoother >= 1) {
      if ((rc = gnn_prepare(c))) return rc;
      sg::k_fcg_scale<float><<<G, B, 0, s>>>(sm, f.r, c->g_rsd.as<float>(),
                                            c->part.as<double>(), c->lanes.as<Lane>());
      gnn_build<float>(c, f.r);
      c->launches++;
      if (mg_on(c) && c->mg_smoother == 2) {  // learned Jacobi weights q^2
        mg::k_mg_square<<<grid_for(c, N), B, 0, s>>>(N, c->g_q.as<float>(), c->mg_dq.as<float>());
        c->launches++;
      }
    }
    if (mg_on(c) && (rc = mg_values(c))) return rc;
    if (mg_on(c) && c->mg_smoother == 1) {
      double f = 1.0;
      if ((rc = mg_bound_smoother(c, &f))) return rc;
      c->mg_smooth_scale = f;
    }
  } else if (imat <= 0) {
    sg::k_cg_rz<float, V, true><<<G, B, 0, s>>>(sm, f.c, f.r, f.z, c->part.as<double>(),
                                                c->lanes.as<Lane>());
    c->launches++;
  }
  CUDA_TRY(c, cudaGetLastError());
  int updates = 0, gl_total = 0, launched = 0;
  // The learned preconditioner hands over to Jacobi-PCG, from the current
  // iterate, when it loses positive curvature or produces NaN (the lane
  // reports kLaneStall), when its residual stalls -- fcg_stall_iters
  // iterations without the residual falling below fcg_stall_drop times its
  // value at the start of that window -- or when the FP64 residual stops
  // improving across reliable updates.
  int cur = solver;
  int imat_cur = imat;  // the hand-over may bring in the DIC/DILU factorisation
  // the residual drop between reliable updates: the learned FCG's own, or
  // (after a hand-over, and for CG) the CG one
  auto delta_of = [&]() { return cur == 2 ? c->fcg_reliable_delta : c->reliable_delta; };
  // after a hand-over: restart the direction (it may hold NaN) and, when
  // asked for, factorise for the reference's DIC/DILU-PCG
  auto restart_fallback = [&]() -> int {
    CUDA_TRY(c, cudaMemsetAsync(f.p, 0, NV * sizeof(float), s));
    CUDA_TRY(c, cudaMemsetAsync(f.q, 0, NV * sizeof(float), s));
    if (imat_cur <= 0 && c->fcg_fallback_imat > 0) {
      int r = launch_precond(c, c->fcg_fallback_imat, w.c, w.cr);
      if (r) return r;
      sg::k_convert<double, float><<<grid_for(c, N), c->block, 0, s>>>(N, w.c, f.c);
      sg::k_convert<double, float><<<grid_for(c, N), c->block, 0, s>>>(N, w.cr, f.cr);
      c->launches += 2;
      imat_cur = c->fcg_fallback_imat;
    }
    return SOLV_GPU_OK;
  };
  c->fallbacks = 0;
  c->smoother_switches = 0;
  // a network smoother that needs more than fcg_slow_iters iterations for
  // one reliable-update drop (the Jacobi-smoothed V-cycle needs about 5 on
  // the systems measured) gives way to damped Jacobi for the rest of the
  // solve, the hierarchy kept
  const int smoother_keep = c->mg_smoother;
  struct SmootherKeep {  // restored on every way out
    solv_gpu_ctx* c;
    int m;
    ~SmootherKeep() { c->mg_smoother = m; }
  } smoother_keep_guard{c, smoother_keep};
  std::vector<int> upd_iter(nl, 0);
  bool switch_smoother = false;
  std::vector<int> win_iter(nl, 0);
  std::vector<double> win_l1(l1_last);
  bool fell_back = false;
  auto hand_over = [&]() {
    if (cur != 2) return;
    cur = 0;
    fell_back = true;
    c->fallbacks++;
  };
  const int K = std::max(1, c->graph_iters);
  while (na > 0) {
    int gl = 0;
    if ((rc = iterate<float, V>(c, cur, imat_cur, K, f, gl))) return rc;  // K iterations at most
    gl_total += gl;
    launched += K;
    CUDA_TRY(c, cudaMemcpyAsync(hl.data(), c->lanes.p, nl * sizeof(Lane), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(c, cudaStreamSynchronize(s));
    bool need = false;
    fell_back = false;
    std::vector<char> trig(nl, 0);
    for (int l = 0; l < nl; ++l) {
      if (final_[l]) continue;
      if (!hl[l].active || hl[l].l1 < delta_of() * l1_last[l]) need = trig[l] = 1;
      if (cur != 2) continue;
      if (hl[l].status == sg::kLaneStall) {
        hand_over();  // no positive curvature from the network
      } else if (hl[l].l1 <= c->fcg_stall_drop * win_l1[l]) {
        win_iter[l] = hl[l].iter;  // progress: a new window starts here
        win_l1[l] = hl[l].l1;
      } else if (hl[l].iter - win_iter[l] >= c->fcg_stall_iters) {
        hand_over();  // the residual stalled
        need = trig[l] = 1;
      }
    }
    if (fell_back && (rc = restart_fallback())) return rc;
    if (!need && launched <= n_iter + K) continue;
    // reliable update of every lane still in play
    for (int l = 0; l < nl; ++l) mask[l] = !final_[l];
    CUDA_TRY(c, cudaMemcpyAsync(c->mp_mask.p, mask.data(), nl * sizeof(int), cudaMemcpyHostToDevice, s));
    sg::k_mp_flush<V><<<G, B, 0, s>>>(sm, c->mp_mask.as<int>(), w.phi, f.phi);
    CUDA_TRY(c, cudaMemcpyAsync(w.r, b, NV * sizeof(double), cudaMemcpyDeviceToDevice, s));
    if ((rc = run_res(c, V, w.phi, w.r, 0))) return rc;
    sg::k_mp_replace<V><<<G, B, 0, s>>>(sm, c->mp_mask.as<int>(), w.r, f.r);
    c->launches += 3;
    ++updates;
    CUDA_TRY(c, cudaMemcpyAsync(l1.data(), c->l1.p, nl * sizeof(double), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(c, cudaStreamSynchronize(s));
    na = 0;
    for (int l = 0; l < nl; ++l) {
      if (final_[l]) {
        hl[l].active = 0;
        continue;
      }
      Lane& L = hl[l];
      ratio[l] = l1[l] / (res0_n[l] + sg::kSmall);
      L.l1 = l1[l];
      L.status = sg::kLaneRunning;
      L.active = 1;
      if (!(ratio[l] == ratio[l]) || std::isinf(ratio[l]) || hl[l].status == sg::kLaneNaN) {
        final_[l] = 1;
        status_v[l] = sg::kLaneNaN;
      } else if (ratio[l] < reduc) {
        final_[l] = 1;
        status_v[l] = sg::kLaneConverged;
      } else if (L.iter >= n_iter || launched > n_iter + K) {
        final_[l] = 1;
        status_v[l] = sg::kLaneMaxIter;
      } else if (trig[l]) {
        // this lane asked for the update but its FP64 residual did not
        // improve on the last one it asked for: FP32 floor, or, for the
        // learned preconditioner, a stall that Jacobi-PCG takes over
        stalls[l] = l1[l] > 0.9 * l1_last[l] ? stalls[l] + 1 : 0;
        if (stalls[l] >= 3 && cur == 2) {
          hand_over();
          stalls[l] = 0;
        } else if (stalls[l] >= 3) {
          final_[l] = 1;
          status_v[l] = sg::kLaneMaxIter;
        }
      }
      if (trig[l] && cur == 2 && !final_[l] && c->mg_smoother >= 1 && mg_on(c) &&
          c->fcg_slow_iters > 0 && L.iter - upd_iter[l] > c->fcg_slow_iters)
        switch_smoother = true;
      if (trig[l]) upd_iter[l] = L.iter;
      if (final_[l]) L.active = 0;
      if (trig[l]) l1_last[l] = l1[l];  // lanes along for the ride keep their window
      L.l1_stop = cur == 2 ? delta_of() * l1_last[l] : 0.0;
      win_iter[l] = L.iter;  // the stall window restarts from the FP64 residual
      win_l1[l] = l1[l];
      na += L.active;
    }
    if (fell_back && (rc = restart_fallback())) return rc;
    if (switch_smoother && cur == 2 && c->mg_smoother >= 1) {
      c->mg_smoother = 0;  // the next iterate() takes the Jacobi-smoothed graph
      c->smoother_switches++;
      CUDA_TRY(c, cudaMemsetAsync(f.p, 0, NV * sizeof(float), s));
      CUDA_TRY(c, cudaMemsetAsync(f.q, 0, NV * sizeof(float), s));
    }
    switch_smoother = false;
    CUDA_TRY(c, cudaMemcpyAsync(c->lanes.p, hl.data(), nl * sizeof(Lane), cudaMemcpyHostToDevice, s));
    CUDA_TRY(c, cudaMemcpyAsync(c->n_active.p, &na, sizeof(int), cudaMemcpyHostToDevice, s));
    if (na == 0) break;
    // The next direction p = z + beta p takes z from the replaced residual,
    // so beta = -(z.q)/(p.q) must too.  The fused Jacobi CG computed it in
    // k_cg_update from the recursive residual: recompute it from the new
    // one, which is the residual the next step works on.  FCG and the
    // sweep-preconditioned CG take beta
    // from the current z already; alpha always comes from p.r of the next
    // step.
    if (cur == 0 && imat_cur <= 0) {
      sg::k_cg_rz<float, V, true, true><<<G, B, 0, s>>>(sm, f.c, f.r, f.z, c->part.as<double>(),
                                                        c->lanes.as<Lane>(), f.q);
      c->launches++;
    }
    CUDA_TRY(c, cudaGetLastError());
  }
  // the caller's check of the sweeps' waits covers its own imat only
  if (imat_cur > 0 && imat <= 0 && (rc = sweep_check(c))) return rc;
  if (not_r0) {
    sg::k_add<<<grid_for(c, NV), c->block, 0, s>>>(NV, w.phi, w.v);
    c->launches++;
  }
  sg::k_phi_out<double><<<grid_for(c, N), c->block, 0, s>>>(N, V, o2n, w.phi, phi_dev);
  c->launches++;
  CUDA_TRY(c, cudaGetLastError());
  int status = SOLV_GPU_OK;
  for (int l = 0; l < nl; ++l) {
    if (status_v[l] == sg::kLaneNaN) status = SOLV_GPU_NAN;
    else if (status_v[l] != sg::kLaneConverged && status == SOLV_GPU_OK) status = SOLV_GPU_MAXITER;
    if (out_iters) out_iters[l] = hl[l].iter;
    if (out_ratio) out_ratio[l] = ratio[l];
  }
  if (st) {
    for (int v = 0; v < V && v < nl; ++v) {
      st->iters[v] = hl[v].iter;
      st->ratio[v] = ratio[v];
    }
    st->status = status;
    st->refinements = updates;
    st->fallbacks = c->fallbacks;
    st->smoother_switches = c->smoother_switches;
    st->mg_levels = solver == 2 && mg_on(c) ? (int)c->mg.size() : 0;
    st->graph_launches += gl_total;
  }
  return status;
}

int solve_dispatch(solv_gpu_ctx* c, int solver, int imat, double reduc, int n_iter, int V,
                   double* phi_dev, double* res0_dev, double* res0_n, int not_r0,
                   solv_gpu_stats* st, int* out_iters, double* out_ratio);

// Device time per launch of the kernels that dominate the solves, each
// launched `repeat` times back to back on workspace vectors (CUDA events on
// the context's stream):
//   4 k_mg_resid       level-0 residual t = b - A x of the V-cycle (FP32)
//   5 k_mg_net<false>  the network's smoothing step x = w K b (FP32)
//   6 k_fcg_spmv       flexible-CG product q = A p with p.q and p.r (FP32)
//   7 k_cg_spmv        FP64 CG product q = A p with p.q (the plain PCG's)
//   8 one DILU application z = M^-1 r, forward + backward recurrence (FP64)
int kernel_time_solve(solv_gpu_ctx* c, int which, int repeat, float* ms_per_launch) {
  const int N = c->N;
  cudaStream_t s = c->stream;
  int rc;
  if (c->n_seg != 1) return set_err(c, SOLV_GPU_BAD_INPUT, "kernel_time: one system only");
  std::function<int()> launch;
  WS<double> w;
  WS<float> f;
  if ((rc = ensure_ws<double>(c, 1, w)) || (rc = ensure_ws<float>(c, 1, f)) ||
      (rc = ensure_f32_matrix(c)))
    return rc;
  sg::k_mp_start<1><<<grid_for(c, N), c->block, 0, s>>>(N, c->diag.as<double>(), f.r, f.p, f.q);
  sg::k_mp_start<1><<<grid_for(c, N), c->block, 0, s>>>(N, c->diag.as<double>(), f.z, f.v, f.phi);
  CUDA_TRY(c, cudaMemcpyAsync(w.p, c->diag.p, N * sizeof(double), cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(c, cudaMemcpyAsync(w.r, c->diag.p, N * sizeof(double), cudaMemcpyDeviceToDevice, s));
  SegMap sm = segmap(c);
  {
    Lane L{};
    L.active = 1;
    L.n_iter = 1 << 30;
    L.reduc = 0.0;
    L.res0_n = 1.0;
    L.s = 1.0;
    L.gs = 1.0;
    const int one = 1;
    CUDA_TRY(c, cudaMemcpyAsync(c->lanes.p, &L, sizeof(Lane), cudaMemcpyHostToDevice, s));
    CUDA_TRY(c, cudaMemcpyAsync(c->n_active.p, &one, sizeof(int), cudaMemcpyHostToDevice, s));
  }
  const int G = c->seg.total_blk, B = c->block;
  double* part = c->part.as<double>();
  Lane* lanes = c->lanes.as<Lane>();
  if (which == 4) {
    launch = [&]() {
      with_chunk(c->row_chunk, [&](auto cc) {
        mg::k_mg_resid<decltype(cc)::value><<<grid_resident(c, N), B, 0, s>>>(N, rows<float>(c), f.r,
                                                                             f.p, f.q, nullptr);
      });
      return SOLV_GPU_OK;
    };
  } else if (which == 5) {
    if ((rc = gnn_prepare(c))) return rc;
    gnn_build<float>(c, f.r);
    launch = [&]() {
      mg::k_mg_net<false, float><<<grid_resident(c, N), B, 0, s>>>(
          N, rows<float>(c), c->g_ge.as<float>(), c->g_q.as<float>(), (float)c->mg_omega, f.r,
          nullptr, f.q, nullptr);
      return SOLV_GPU_OK;
    };
  } else if (which == 6) {
    launch = [&]() {
      with_chunk(c->row_chunk, [&](auto cc) {
        sg::k_fcg_spmv<float, decltype(cc)::value><<<G, B, 0, s>>>(rows<float>(c), sm, f.p, f.q,
                                                                   f.r, part, lanes);
      });
      return SOLV_GPU_OK;
    };
  } else if (which == 7) {
    launch = [&]() {
      sg::k_cg_spmv<double, 1><<<G, B, 0, s>>>(rows<double>(c), sm, w.p, w.q, part, lanes);
      return SOLV_GPU_OK;
    };
  } else {
    if ((rc = launch_precond(c, 2, w.c, w.cr))) return rc;
    launch = [&]() { return launch_direct<double, 1>(c, 2, w.c, w.cr, w.z, w.r, nullptr); };
  }
  if ((rc = launch())) return rc;
  CUDA_TRY(c, cudaEventRecord(c->ev0, s));
  for (int k = 0; k < repeat; ++k)
    if ((rc = launch())) return rc;
  CUDA_TRY(c, cudaEventRecord(c->ev1, s));
  CUDA_TRY(c, cudaEventSynchronize(c->ev1));
  CUDA_TRY(c, cudaGetLastError());
  if (which == 8 && (rc = sweep_check(c))) return rc;
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  *ms_per_launch = ms / repeat;
  return SOLV_GPU_OK;
}

}  // namespace

// =============================== C-ABI ========================================
extern "C" {

const char* solv_gpu_status_string(int s) {
  switch (s) {
    case SOLV_GPU_OK: return "ok";
    case SOLV_GPU_MAXITER: return "iteration cap reached";
    case SOLV_GPU_NAN: return "NaN/Inf in a reduction";
    case SOLV_GPU_BAD_INPUT: return "bad input";
    case SOLV_GPU_DEVICE_ERROR: return "CUDA error";
    case SOLV_GPU_NO_MATRIX: return "no matrix set";
    case SOLV_GPU_ZERO_RHS: return "zero initial residual (early return)";
    case SOLV_GPU_TOO_LARGE: return "problem larger than the fixed scratch";
    case SOLV_GPU_TIMEOUT: return "a bounded device wait ran out";
    default: return "unknown status";
  }
}

const char* solv_gpu_last_error(const solv_gpu_ctx* c) { return c ? c->err.c_str() : "null context"; }

int solv_gpu_create(solv_gpu_ctx** out, int device) {
  if (!out) return SOLV_GPU_BAD_INPUT;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return SOLV_GPU_DEVICE_ERROR;
  if (device < 0 || device >= ndev) return SOLV_GPU_BAD_INPUT;
  auto* c = new solv_gpu_ctx();
  c->dev = device;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMallocHost(&c->h_n_active, 2 * sizeof(int)) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
    delete c;
    return SOLV_GPU_DEVICE_ERROR;
  }
  c->stream = c->own;
  cudaDeviceGetAttribute(&c->n_sm, cudaDevAttrMultiProcessorCount, device);
  *out = c;
  return SOLV_GPU_OK;
}

int solv_gpu_destroy(solv_gpu_ctx* c) {
  if (!c) return SOLV_GPU_BAD_INPUT;
  cudaSetDevice(c->dev);
  cudaStreamSynchronize(c->stream);
  drop_graphs(c);
  if (c->h_n_active) cudaFreeHost(c->h_n_active);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  cudaStream_t own = c->own;
  delete c;  // DevBufs free their memory
  if (own) cudaStreamDestroy(own);
  return SOLV_GPU_OK;
}

int solv_gpu_set_stream(solv_gpu_ctx* c, void* stream) {
  if (!c) return SOLV_GPU_BAD_INPUT;
  cudaStream_t s = stream ? (cudaStream_t)stream : c->own;
  if (s != c->stream) {
    drop_graphs(c);
    c->stream = s;
  }
  return SOLV_GPU_OK;
}

int solv_gpu_set_option(solv_gpu_ctx* c, int key, double value) {
  if (!c) return SOLV_GPU_BAD_INPUT;
  switch (key) {
    case SOLV_OPT_PRECISION:
      if (value != 0 && value != 1) return set_err(c, SOLV_GPU_BAD_INPUT, "precision must be 0 or 1");
      c->precision = (int)value;
      return SOLV_GPU_OK;
    case SOLV_OPT_INNER_REDUC:
      if (!(value > 0 && value < 1)) return set_err(c, SOLV_GPU_BAD_INPUT, "inner reduc must be in (0,1)");
      c->inner_reduc = value;
      return SOLV_GPU_OK;
    case SOLV_OPT_GRAPH_ITERS:
      if (value < 0 || value > 1024) return set_err(c, SOLV_GPU_BAD_INPUT, "graph iters in 0..1024");
      c->graph_iters = (int)value;
      drop_graphs(c);
      return SOLV_GPU_OK;
    case SOLV_OPT_BLOCK: {
      int b = (int)value;
      if (b < 64 || b > sg::kMaxBlock || (b & 31))
        return set_err(c, SOLV_GPU_BAD_INPUT, "block must be a multiple of 32 in 64..256");
      c->block = b;
      if (c->has_matrix) return build_segments(c, c->seg_c0_caller, c->seg_c1_caller);
      return SOLV_GPU_OK;
    }
    case SOLV_OPT_GRID_PER_SM: {
      int g = (int)value;
      if (g < 1 || g > 64) return set_err(c, SOLV_GPU_BAD_INPUT, "grid per SM in 1..64");
      c->grid_per_sm = g;
      if (c->has_matrix) return build_segments(c, c->seg_c0_caller, c->seg_c1_caller);
      return SOLV_GPU_OK;
    }
    case SOLV_OPT_MAX_REFINE:
      if (value < 1 || value > 1000) return set_err(c, SOLV_GPU_BAD_INPUT, "max refine in 1..1000");
      c->max_refine = (int)value;
      return SOLV_GPU_OK;
    case SOLV_OPT_GNN_LOSS:
      if (value != 0 && value != 1 && value != 2)
        return set_err(c, SOLV_GPU_BAD_INPUT, "gnn loss is 0, 1 or 2");
      c->gnn_loss = (int)value;
      return SOLV_GPU_OK;
    case SOLV_OPT_RELIABLE_DELTA:
      if (!(value > 0 && value < 1)) return set_err(c, SOLV_GPU_BAD_INPUT, "reliable delta in (0,1)");
      c->reliable_delta = value;
      return SOLV_GPU_OK;
    case SOLV_OPT_GRAPH_LOOP:
      if (value != 0 && value != 1 && value != 2)
        return set_err(c, SOLV_GPU_BAD_INPUT, "graph loop is 0, 1 or 2");
      c->graph_loop = (int)value;
      return SOLV_GPU_OK;
    case SOLV_OPT_FCG_SLOW_ITERS:
      if (value < 0 || value > 1e7) return set_err(c, SOLV_GPU_BAD_INPUT, "slow-iteration limit in 0..1e7");
      c->fcg_slow_iters = (int)value;
      return SOLV_GPU_OK;
    case SOLV_OPT_FCG_FALLBACK:
      if (value != 0 && value != 1 && value != 2)
        return set_err(c, SOLV_GPU_BAD_INPUT, "fallback preconditioner is 0, 1 or 2");
      c->fcg_fallback_imat = (int)value;
      return SOLV_GPU_OK;
    case SOLV_OPT_FCG_RELIABLE_DELTA:
      if (!(value > 0 && value < 1))
        return set_err(c, SOLV_GPU_BAD_INPUT, "reliable delta in (0,1)");
      c->fcg_reliable_delta = value;
      return SOLV_GPU_OK;
    case SOLV_OPT_MG_LEVELS:  // 0 keeps a built hierarchy aside; another maximum rebuilds it
      if (value < 0 || value > mg::kMaxLevels)
        return set_err(c, SOLV_GPU_BAD_INPUT, "multigrid levels in 0..12");
      if ((int)value != c->mg_max_levels) {
        c->mg_max_levels = (int)value;
        drop_graphs(c);
      }
      return SOLV_GPU_OK;
    case SOLV_OPT_MG_SMOOTHER:
      if (value != 0 && value != 1 && value != 2)
        return set_err(c, SOLV_GPU_BAD_INPUT, "multigrid smoother is 0, 1 or 2");
      if ((int)value != c->mg_smoother) {
        c->mg_smoother = (int)value;
        drop_graphs(c);
      }
      return SOLV_GPU_OK;
    case SOLV_OPT_MG_OMEGA:
      if (!(value > 0 && value < 2)) return set_err(c, SOLV_GPU_BAD_INPUT, "smoother damping in (0,2)");
      if (value != c->mg_omega) {
        c->mg_omega = value;
        drop_graphs(c);
      }
      return SOLV_GPU_OK;
    case SOLV_OPT_MG_ALPHA:
      if (!(value > 0 && value <= 4)) return set_err(c, SOLV_GPU_BAD_INPUT, "coarse-correction scale in (0,4]");
      if (value != c->mg_alpha) {
        c->mg_alpha = value;
        drop_graphs(c);
      }
      return SOLV_GPU_OK;
    case SOLV_OPT_FCG_STALL_ITERS:
      if (value < 1 || value > 1e7) return set_err(c, SOLV_GPU_BAD_INPUT, "stall window in 1..1e7");
      c->fcg_stall_iters = (int)value;
      return SOLV_GPU_OK;
    case SOLV_OPT_FCG_STALL_DROP:
      if (!(value > 0 && value < 1)) return set_err(c, SOLV_GPU_BAD_INPUT, "stall drop in (0,1)");
      c->fcg_stall_drop = value;
      return SOLV_GPU_OK;
    case SOLV_OPT_MG_SCALE_MIN:
      if (!(value >= 0 && value <= 1)) return set_err(c, SOLV_GPU_BAD_INPUT, "scale floor in [0,1]");
      c->mg_scale_min = (float)value;
      return SOLV_GPU_OK;
    case SOLV_OPT_PERSISTENT:
      if (value != 0 && value != 1) return set_err(c, SOLV_GPU_BAD_INPUT, "persistent is 0 or 1");
      c->persistent = (int)value;
      return SOLV_GPU_OK;
    case SOLV_OPT_VECTOR_WIDTH:
      if (value != 2 && value != 4 && value != 8)
        return set_err(c, SOLV_GPU_BAD_INPUT, "vector width is 2, 4 or 8");
      if ((int)value != c->row_chunk) {
        c->row_chunk = (int)value;
        drop_graphs(c);
      }
      return SOLV_GPU_OK;
    case SOLV_OPT_MG_BUILD:
      if (value != 0 && value != 1) return set_err(c, SOLV_GPU_BAD_INPUT, "hierarchy build is 0 or 1");
      if ((int)value != c->mg_build) {
        c->mg_build = (int)value;
        c->mg_valid = false;
        drop_graphs(c);
      }
      return SOLV_GPU_OK;
    case SOLV_OPT_INNER_MAX_ITER:
      if (value < 1 || value > 1e7) return set_err(c, SOLV_GPU_BAD_INPUT, "inner max iter in 1..1e7");
      c->inner_max_iter = (int)value;
      return SOLV_GPU_OK;
    default:
      return set_err(c, SOLV_GPU_BAD_INPUT, "unknown option key");
  }
}

int solv_gpu_matrix_set(solv_gpu_ctx* c, int n_cell, int n_face, const int* ip, const int* in,
                        const double* p, const double* n, const double* pl) {
  if (!c) return SOLV_GPU_BAD_INPUT;
  if (!p || !n || !pl) return set_err(c, SOLV_GPU_BAD_INPUT, "matrix_set: null coefficient pointer");
  CUDA_TRY(c, cudaSetDevice(c->dev));
  c->has_matrix = false;
  int rc = matrix_structure(c, n_cell, n_face, ip, in, 1, nullptr);
  if (rc) return rc;
  return solv_gpu_matrix_values(c, p, n, pl);
}

int solv_gpu_matrix_values(solv_gpu_ctx* c, const double* p, const double* n, const double* pl) {
  if (!c) return SOLV_GPU_BAD_INPUT;
  if (!c->has_matrix) return set_err(c, SOLV_GPU_NO_MATRIX, "no matrix set");
  if (!p || !n || !pl) return set_err(c, SOLV_GPU_BAD_INPUT, "matrix_values: null pointer");
  CUDA_TRY(c, cudaSetDevice(c->dev));
  CUDA_TRY(c, c->w_in.ensure((size_t)c->N * sizeof(double)));
  if (c->F > 0) {
    CUDA_TRY(c, cudaMemcpyAsync(c->fp.p, p, c->F * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(c->fn.p, n, c->F * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  }
  CUDA_TRY(c, cudaMemcpyAsync(c->w_in.p, pl, c->N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  int rc = matrix_values_dev(c, c->fp.as<double>(), c->fn.as<double>(), c->w_in.as<double>());
  if (rc) return rc;
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return SOLV_GPU_OK;
}

int solv_gpu_matrix_values_dev(solv_gpu_ctx* c, const double* p, const double* n, const double* pl) {
  if (!c) return SOLV_GPU_BAD_INPUT;
  if (!p || !n || !pl) return set_err(c, SOLV_GPU_BAD_INPUT, "matrix_values_dev: null pointer");
  CUDA_TRY(c, cudaSetDevice(c->dev));
  return matrix_values_dev(c, p, n, pl);
}

int solv_gpu_matrix_levels(const solv_gpu_ctx* c) {
  if (!c || !c->has_matrix) return -1;
  return (int)c->lvl_ptr.size() - 1;
}

int solv_gpu_res(solv_gpu_ctx* c, int n_vc, const double* phi, double* res0, double* res0_n,
                 int not_r0) {
  if (!c) return SOLV_GPU_BAD_INPUT;
  if (!c->has_matrix) return set_err(c, SOLV_GPU_NO_MATRIX, "no matrix set");
  if (n_vc < 1 || n_vc > kMaxV || !phi || !res0 || !res0_n)
    return set_err(c, SOLV_GPU_BAD_INPUT, "res: n_vc must be 1..4 and pointers non-null");
  CUDA_TRY(c, cudaSetDevice(c->dev));
  const int N = c->N, V = n_vc;
  const size_t bytes = (size_t)N * V * sizeof(double);
  CUDA_TRY(c, c->w_in.ensure(bytes));
  CUDA_TRY(c, c->w_out.ensure(bytes));
  CUDA_TRY(c, c->w_x.ensure(bytes));
  CUDA_TRY(c, c->w_b.ensure(bytes));
  cudaStream_t s = c->stream;
  const int* o2n = c->old_of_new.as<int>();
  CUDA_TRY(c, cudaMemcpyAsync(c->w_in.p, phi, bytes, cudaMemcpyHostToDevice, s));
  CUDA_TRY(c, cudaMemcpyAsync(c->w_out.p, res0, bytes, cudaMemcpyHostToDevice, s));
  sg::k_phi_in<double><<<grid_for(c, N), c->block, 0, s>>>(N, V, o2n, c->w_in.as<double>(), c->w_x.as<double>());
  sg::k_col_in<<<grid_for(c, N), c->block, 0, s>>>(N, V, o2n, c->w_out.as<double>(), c->w_b.as<double>());
  int rc = run_res(c, V, c->w_x.as<double>(), c->w_b.as<double>(), not_r0);
  if (rc) return rc;
  sg::k_col_out<<<grid_for(c, N), c->block, 0, s>>>(N, V, o2n, c->w_b.as<double>(), c->w_out.as<double>());
  CUDA_TRY(c, cudaMemcpyAsync(res0, c->w_out.p, bytes, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(c, cudaMemcpyAsync(res0_n, c->l1.p, V * sizeof(double), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(c, cudaStreamSynchronize(s));
  return SOLV_GPU_OK;
}

int solv_gpu_precond(solv_gpu_ctx* c, int imat, double* cc, double* cr) {
  if (!c) return SOLV_GPU_BAD_INPUT;
  if (!c->has_matrix) return set_err(c, SOLV_GPU_NO_MATRIX, "no matrix set");
  if (!cc || !cr) return set_err(c, SOLV_GPU_BAD_INPUT, "precond: null pointer");
  CUDA_TRY(c, cudaSetDevice(c->dev));
  const int N = c->N;
  const size_t bytes = (size_t)N * sizeof(double);
  CUDA_TRY(c, c->w_x.ensure(bytes));
  CUDA_TRY(c, c->w_b.ensure(bytes));
  CUDA_TRY(c, c->w_out.ensure(bytes));
  cudaStream_t s = c->stream;
  const int* o2n = c->old_of_new.as<int>();
  {
    WS<double> w;  // the sweep state, allocated with the workspace
    int rc = ensure_ws<double>(c, 1, w);
    if (rc || (rc = launch_precond(c, imat, c->w_x.as<double>(), c->w_b.as<double>())) ||
        (rc = sweep_check(c)))
      return rc;
  }
  sg::k_phi_out<double><<<grid_for(c, N), c->block, 0, s>>>(N, 1, o2n, c->w_x.as<double>(), c->w_out.as<double>());
  CUDA_TRY(c, cudaMemcpyAsync(cc, c->w_out.p, bytes, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(c, cudaStreamSynchronize(s));
  sg::k_phi_out<double><<<grid_for(c, N), c->block, 0, s>>>(N, 1, o2n, c->w_b.as<double>(), c->w_out.as<double>());
  CUDA_TRY(c, cudaMemcpyAsync(cr, c->w_out.p, bytes, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(c, cudaStreamSynchronize(s));
  CUDA_TRY(c, cudaGetLastError());
  return SOLV_GPU_OK;
}

int solv_gpu_direct(solv_gpu_ctx* c, int imat, const double* cc, const double* cr, double* x,
                    const double* b) {
  if (!c) return SOLV_GPU_BAD_INPUT;
  if (!c->has_matrix) return set_err(c, SOLV_GPU_NO_MATRIX, "no matrix set");
  if (!cc || !cr || !x || !b) return set_err(c, SOLV_GPU_BAD_INPUT, "direct: null pointer");
  CUDA_TRY(c, cudaSetDevice(c->dev));
  const int N = c->N;
  const size_t bytes = (size_t)N * sizeof(double);
  WS<double> w;
  int rc = ensure_ws<double>(c, 1, w);
  if (rc) return rc;
  CUDA_TRY(c, c->w_in.ensure(bytes));
  cudaStream_t s = c->stream;
  const int* o2n = c->old_of_new.as<int>();
  auto up = [&](const double* h, double* d) -> int {
    CUDA_TRY(c, cudaMemcpyAsync(c->w_in.p, h, bytes, cudaMemcpyHostToDevice, s));
    sg::k_phi_in<double><<<grid_for(c, N), c->block, 0, s>>>(N, 1, o2n, c->w_in.as<double>(), d);
    return SOLV_GPU_OK;
  };
  if ((rc = up(cc, w.c)) || (rc = up(cr, w.cr)) || (rc = up(b, w.r))) return rc;
  if ((rc = launch_direct<double, 1>(c, imat, w.c, w.cr, w.z, w.r, nullptr)) ||
      (rc = sweep_check(c)))
    return rc;
  sg::k_phi_out<double><<<grid_for(c, N), c->block, 0, s>>>(N, 1, o2n, w.z, c->w_in.as<double>());
  CUDA_TRY(c, cudaMemcpyAsync(x, c->w_in.p, bytes, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(c, cudaStreamSynchronize(s));
  CUDA_TRY(c, cudaGetLastError());
  return SOLV_GPU_OK;
}

int solv_gpu_spmv_dev(solv_gpu_ctx* c, const double* x_dev, double* y_dev, int repeat,
                      float* ms_per_call) {
  if (!c) return SOLV_GPU_BAD_INPUT;
  if (!c->has_matrix) return set_err(c, SOLV_GPU_NO_MATRIX, "no matrix set");
  CUDA_TRY(c, cudaSetDevice(c->dev));
  const int N = c->N;
  const size_t bytes = (size_t)N * sizeof(double);
  CUDA_TRY(c, c->w_x.ensure(bytes));
  CUDA_TRY(c, c->w_b.ensure(bytes));
  cudaStream_t s = c->stream;
  const int* o2n = c->old_of_new.as<int>();
  sg::k_phi_in<double><<<grid_for(c, N), c->block, 0, s>>>(N, 1, o2n, x_dev, c->w_x.as<double>());
  if (repeat < 1) repeat = 1;
  CUDA_TRY(c, cudaEventRecord(c->ev0, s));
  for (int k = 0; k < repeat; ++k)
    sg::k_spmv<double, 1><<<grid_resident(c, N), c->block, 0, s>>>(N, rows<double>(c), c->w_x.as<double>(),
                                                                c->w_b.as<double>());
  CUDA_TRY(c, cudaEventRecord(c->ev1, s));
  sg::k_phi_out<double><<<grid_for(c, N), c->block, 0, s>>>(N, 1, o2n, c->w_b.as<double>(), y_dev);
  CUDA_TRY(c, cudaStreamSynchronize(s));
  CUDA_TRY(c, cudaGetLastError());
  if (ms_per_call) {
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    *ms_per_call = ms / repeat;
  }
  return SOLV_GPU_OK;
}

// Device time of one kernel of the solve path, timed with events on the
// context's stream over `repeat` back-to-back launches on workspace vectors:
// which 0 = FP64 matrix product, 1 = FP32 matrix product, 2 = the learned
// preconditioner's application (FP32; needs parameters, builds M^-1 from a
// constant residual first).
int solv_gpu_selftest_sweep_wait(solv_gpu_ctx* c) {
  if (!c) return SOLV_GPU_BAD_INPUT;
  CUDA_TRY(c, cudaSetDevice(c->dev));
  DevBuf w, v;
  CUDA_TRY(c, w.ensure(16));
  CUDA_TRY(c, v.ensure(sizeof(double)));
  if (!c->sweep_ctl.p) {
    CUDA_TRY(c, c->sweep_ctl.ensure(sizeof(sg::SweepCtl)));
    CUDA_TRY(c, cudaMemsetAsync(c->sweep_ctl.p, 0, sizeof(sg::SweepCtl), c->stream));
  }
  const uint8_t one = 1;
  CUDA_TRY(c, cudaMemcpyAsync(w.p, &one, 1, cudaMemcpyHostToDevice, c->stream));
  sg::k_fill_pending<double><<<1, 32, 0, c->stream>>>(1, v.as<double>());
  sg::k_sweep_selftest<<<1, 32, 0, c->stream>>>(w.as<uint8_t>(), v.as<double>(), sweep_ctl(c));
  CUDA_TRY(c, cudaGetLastError());
  return sweep_check(c);  // synchronises; SOLV_GPU_TIMEOUT when the wait ran out
}

int solv_gpu_kernel_time(solv_gpu_ctx* c, int which, int repeat, float* ms_per_launch) {
  if (!c) return SOLV_GPU_BAD_INPUT;
  if (!c->has_matrix) return set_err(c, SOLV_GPU_NO_MATRIX, "no matrix set");
  if (which < 0 || which > 8 || repeat < 1 || !ms_per_launch)
    return set_err(c, SOLV_GPU_BAD_INPUT, "kernel_time: bad arguments");
  CUDA_TRY(c, cudaSetDevice(c->dev));
  const int N = c->N;
  cudaStream_t s = c->stream;
  int rc;
  if (which >= 4) return kernel_time_solve(c, which, repeat, ms_per_launch);
  if (which == 0) {
    WS<double> w;
    if ((rc = ensure_ws<double>(c, 1, w))) return rc;
    CUDA_TRY(c, cudaMemsetAsync(w.p, 0, N * sizeof(double), s));
    sg::k_spmv<double, 1><<<grid_resident(c, N), c->block, 0, s>>>(N, rows<double>(c), w.p, w.q);
    CUDA_TRY(c, cudaEventRecord(c->ev0, s));
    for (int k = 0; k < repeat; ++k)
      sg::k_spmv<double, 1><<<grid_resident(c, N), c->block, 0, s>>>(N, rows<double>(c), w.p, w.q);
    CUDA_TRY(c, cudaEventRecord(c->ev1, s));
  } else {
    WS<float> f;
    if ((rc = ensure_ws<float>(c, 1, f))) return rc;
    if ((rc = ensure_f32_matrix(c))) return rc;
    CUDA_TRY(c, cudaMemsetAsync(f.p, 0, N * sizeof(float), s));
    if (which == 3) {
      if (c->mg_max_levels <= 0) return set_err(c, SOLV_GPU_BAD_INPUT, "kernel_time: multigrid is off");
      if ((rc = mg_setup(c))) return rc;
      if (!mg_on(c)) return set_err(c, SOLV_GPU_BAD_INPUT, "kernel_time: no hierarchy for this matrix");
      if ((rc = mg_values(c))) return rc;
    }
    if (which == 2 || (which == 3 && c->mg_smoother >= 1)) {
      if ((rc = gnn_prepare(c))) return rc;
      Lane L{};
      L.active = 1;
      L.gs = 1.0;
      CUDA_TRY(c, cudaMemcpyAsync(c->lanes.p, &L, sizeof(Lane), cudaMemcpyHostToDevice, s));
      gnn_build<float>(c, f.p);
      if (which == 3 && c->mg_smoother == 2)
        mg::k_mg_square<<<grid_for(c, N), c->block, 0, s>>>(N, c->g_q.as<float>(),
                                                           c->mg_dq.as<float>());
    }
    auto launch = [&]() {
      if (which == 1)
        sg::k_spmv<float, 1><<<grid_resident(c, N), c->block, 0, s>>>(N, rows<float>(c), f.p, f.q);
      else if (which == 2)
        gnn::k_gnn_apply<float><<<grid_for(c, N), c->block, 0, s>>>(
            N, rows<float>(c), c->g_ge.as<float>(), c->g_q.as<float>(), f.p, f.q, nullptr);
      else
        mg_vcycle<float>(c, f.p, f.q, c->mg_smoother, c->g_q.as<float>(),
                         c->g_ge.as<float>(), c->mg_x0.as<float>(), c->mg_t0.as<float>(), nullptr);
    };
    launch();
    CUDA_TRY(c, cudaEventRecord(c->ev0, s));
    for (int k = 0; k < repeat; ++k) launch();
    CUDA_TRY(c, cudaEventRecord(c->ev1, s));
  }
  CUDA_TRY(c, cudaEventSynchronize(c->ev1));
  CUDA_TRY(c, cudaGetLastError());
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev0, c->ev1);
  *ms_per_launch = ms / repeat;
  return SOLV_GPU_OK;
}

int solv_gpu_spmv(solv_gpu_ctx* c, const double* x, double* y) {
  if (!c) return SOLV_GPU_BAD_INPUT;
  if (!c->has_matrix) return set_err(c, SOLV_GPU_NO_MATRIX, "no matrix set");
  if (!x || !y) return set_err(c, SOLV_GPU_BAD_INPUT, "spmv: null pointer");
  CUDA_TRY(c, cudaSetDevice(c->dev));
  const size_t bytes = (size_t)c->N * sizeof(double);
  CUDA_TRY(c, c->w_in.ensure(bytes));
  CUDA_TRY(c, c->w_out.ensure(bytes));
  CUDA_TRY(c, cudaMemcpyAsync(c->w_in.p, x, bytes, cudaMemcpyHostToDevice, c->stream));
  int rc = solv_gpu_spmv_dev(c, c->w_in.as<double>(), c->w_out.as<double>(), 1, nullptr);
  if (rc) return rc;
  CUDA_TRY(c, cudaMemcpyAsync(y, c->w_out.p, bytes, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return SOLV_GPU_OK;
}

static int solve_common(solv_gpu_ctx* c, int solver, int imat, double reduc, int n_iter, int n_vc,
                        double* phi_dev, double* res0_dev, double* res0_n, int not_r0,
                        solv_gpu_stats* st, int* out_iters = nullptr, double* out_ratio = nullptr,
                        bool batch = false) {
  if (!c) return SOLV_GPU_BAD_INPUT;
  if (!c->has_matrix) return set_err(c, SOLV_GPU_NO_MATRIX, "no matrix set");
  if (n_vc < 1 || n_vc > kMaxV) return set_err(c, SOLV_GPU_BAD_INPUT, "n_vc must be 1..4");
  if (imat < 0 || imat > 2) return set_err(c, SOLV_GPU_BAD_INPUT, "imat must be 0, 1 or 2");
  if (!phi_dev || !res0_dev || !res0_n) return set_err(c, SOLV_GPU_BAD_INPUT, "null pointer");
  if (c->n_seg > 1 && !batch)
    return set_err(c, SOLV_GPU_BAD_INPUT, "a batch of systems is set: use the _batch entry points");
  c->err.clear();
  if (st) {
    std::memset(st, 0, sizeof(*st));
    st->n_levels = (int)c->lvl_ptr.size() - 1;
  }
  CUDA_TRY(c, cudaSetDevice(c->dev));
  c->launches = 0;
  CUDA_TRY(c, cudaEventRecord(c->ev0, c->stream));
  int rc = solve_dispatch(c, solver, imat, reduc, n_iter, n_vc, phi_dev, res0_dev, res0_n, not_r0,
                          st, out_iters, out_ratio);
  if (imat > 0 && c->sweep_ctl.p && (rc == SOLV_GPU_OK || rc == SOLV_GPU_MAXITER || rc == SOLV_GPU_NAN)) {
    const int rs = sweep_check(c);
    if (rs) rc = rs;
  }
  CUDA_TRY(c, cudaEventRecord(c->ev1, c->stream));
  CUDA_TRY(c, cudaEventSynchronize(c->ev1));
  if (st) {
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    st->solve_ms = ms;
    st->kernel_launches = c->launches;
    if (rc != SOLV_GPU_OK && rc != SOLV_GPU_MAXITER && rc != SOLV_GPU_NAN) st->status = rc;
  }
  return rc;
}

static int solve_host(solv_gpu_ctx* c, int solver, int imat, double reduc, int n_iter, int n_vc,
                      double* phi, double* res0, double* res0_n, int not_r0, solv_gpu_stats* st,
                      int* out_iters = nullptr, double* out_ratio = nullptr, bool batch = false) {
  if (!c) return SOLV_GPU_BAD_INPUT;
  if (!c->has_matrix) return set_err(c, SOLV_GPU_NO_MATRIX, "no matrix set");
  if (n_vc < 1 || n_vc > kMaxV) return set_err(c, SOLV_GPU_BAD_INPUT, "n_vc must be 1..4");
  if (!phi || !res0 || !res0_n) return set_err(c, SOLV_GPU_BAD_INPUT, "null pointer");
  CUDA_TRY(c, cudaSetDevice(c->dev));
  const size_t bytes = (size_t)c->N * n_vc * sizeof(double);
  CUDA_TRY(c, c->w_in.ensure(bytes));
  CUDA_TRY(c, c->w_out.ensure(bytes));
  CUDA_TRY(c, cudaMemcpyAsync(c->w_in.p, phi, bytes, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(c->w_out.p, res0, bytes, cudaMemcpyHostToDevice, c->stream));
  int rc = solve_common(c, solver, imat, reduc, n_iter, n_vc, c->w_in.as<double>(),
                        c->w_out.as<double>(), res0_n, not_r0, st, out_iters, out_ratio, batch);
  if (rc != SOLV_GPU_OK && rc != SOLV_GPU_MAXITER && rc != SOLV_GPU_NAN) return rc;
  CUDA_TRY(c, cudaMemcpyAsync(phi, c->w_in.p, bytes, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(res0, c->w_out.p, bytes, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return rc;
}

int solv_gpu_cg(solv_gpu_ctx* c, int imat, double reduc, int n_iter, int n_vc, double* phi,
                double* res0, double* res0_n, int not_r0, solv_gpu_stats* st) {
  return solve_host(c, 0, imat, reduc, n_iter, n_vc, phi, res0, res0_n, not_r0, st);
}
int solv_gpu_bicg(solv_gpu_ctx* c, int imat, double reduc, int n_iter, int n_vc, double* phi,
                  double* res0, double* res0_n, int not_r0, solv_gpu_stats* st) {
  return solve_host(c, 1, imat, reduc, n_iter, n_vc, phi, res0, res0_n, not_r0, st);
}
int solv_gpu_cg_dev(solv_gpu_ctx* c, int imat, double reduc, int n_iter, int n_vc, double* phi,
                    double* res0, double* res0_n, int not_r0, solv_gpu_stats* st) {
  return solve_common(c, 0, imat, reduc, n_iter, n_vc, phi, res0, res0_n, not_r0, st);
}
int solv_gpu_bicg_dev(solv_gpu_ctx* c, int imat, double reduc, int n_iter, int n_vc, double* phi,
                      double* res0, double* res0_n, int not_r0, solv_gpu_stats* st) {
  return solve_common(c, 1, imat, reduc, n_iter, n_vc, phi, res0, res0_n, not_r0, st);
}

// ---- autotuner -----------------------------------------------------------------
// Chooses threads per block, resident blocks per SM of the reduction
// kernels, Krylov iterations per CUDA graph and, where the iteration runs in
// FP32 (precision 1, or the learned FCG), the products' vector width (matrix
// slots a thread loads per step) for the current matrix (one system or a
// batch), solver, preconditioner, component count and precision.  Each
// candidate is timed on the device by differencing a short and a long
// capped solve of a seeded right-hand side (so setup and layout conversion
// cancel out); the fastest per-iteration time wins and is left set on the
// context.  The configuration in effect before tuning is timed the same
// way, first, stays eligible, and is reported beside the winner.
int solv_gpu_autotune(solv_gpu_ctx* c, int solver, int imat, int n_vc, solv_gpu_tune* out) {
  if (!c) return SOLV_GPU_BAD_INPUT;
  if (!c->has_matrix) return set_err(c, SOLV_GPU_NO_MATRIX, "no matrix set");
  if (n_vc < 1 || n_vc > kMaxV || imat < 0 || imat > 2 || solver < 0 || solver > 2)
    return set_err(c, SOLV_GPU_BAD_INPUT, "autotune: bad solver / imat / n_vc");
  if (solver == 2 && (n_vc != 1 || c->n_seg != 1 || !c->g_has_params))
    return set_err(c, SOLV_GPU_BAD_INPUT,
                   "autotune: the learned solve needs one system, n_vc = 1 and network parameters");
  CUDA_TRY(c, cudaSetDevice(c->dev));
  const int N = c->N, V = n_vc, nl = c->n_seg * V;
  const size_t nv = (size_t)N * V;
  DevBuf phi, res, b;
  CUDA_TRY(c, phi.ensure(nv * sizeof(double)));
  CUDA_TRY(c, res.ensure(nv * sizeof(double)));
  CUDA_TRY(c, b.ensure(nv * sizeof(double)));
  {
    std::vector<double> hb(nv);
    uint64_t x = 0x9e3779b97f4a7c15ull;
    for (size_t i = 0; i < nv; ++i) {  // splitmix64 -> uniform [-1, 1)
      x += 0x9e3779b97f4a7c15ull;
      uint64_t z = x;
      z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
      z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
      z ^= z >> 31;
      hb[i] = (double)(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    }
    CUDA_TRY(c, cudaMemcpy(b.p, hb.data(), nv * sizeof(double), cudaMemcpyHostToDevice));
  }
  std::vector<double> rn(nl);
  auto run = [&](int iters, float& ms) -> int {
    CUDA_TRY(c, cudaMemsetAsync(phi.p, 0, nv * sizeof(double), c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(res.p, b.p, nv * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    solv_gpu_stats st;
    int rc = solve_common(c, solver, imat, 1e-300, iters, V, phi.as<double>(), res.as<double>(),
                          rn.data(), 0, &st, nullptr, nullptr, true);
    if (rc != SOLV_GPU_OK && rc != SOLV_GPU_MAXITER) return rc;
    ms = (float)st.solve_ms;
    return SOLV_GPU_OK;
  };
  const int k_short = 4, k_long = 36;
  // per-iteration time of the context's current settings
  auto measure = [&](double& per) -> int {
    int rc = build_segments(c, c->seg_c0_caller, c->seg_c1_caller);
    if (rc) return rc;
    float t0 = 0, t1 = 0, w = 0;
    if ((rc = run(k_short, w))) return rc;  // warm: graph capture, workspace
    if ((rc = run(k_short, t0)) || (rc = run(k_long, t1))) return rc;
    per = (t1 - t0) / (double)(k_long - k_short);
    return SOLV_GPU_OK;
  };
  const bool fp32 = c->precision == 1 || solver == 2;
  // the measured iterations are all real work: no lane stops early for a
  // reliable update (it would leave the rest of a graph as early exits)
  struct DeltaKeep {  // restored on every way out
    solv_gpu_ctx* c;
    double d, fd;
    ~DeltaKeep() {
      c->reliable_delta = d;
      c->fcg_reliable_delta = fd;
    }
  } delta_keep{c, c->reliable_delta, c->fcg_reliable_delta};
  c->reliable_delta = c->fcg_reliable_delta = 1e-300;
  const int blocks[] = {128, 256};
  const int gps[] = {4, 8, 16};
  const int graphs[] = {8, 32};
  std::vector<int> widths = fp32 ? std::vector<int>{2, 4, 8} : std::vector<int>{c->row_chunk};
  const int precision = c->precision;
  // the tuner measures capped iterations: keep FP32 sweeps as long as the cap
  const int inner_keep = c->inner_max_iter;
  double per_default = 0.0;
  drop_graphs(c);
  int rc = measure(per_default);
  if (rc) return rc;
  // the settings before the call stay eligible: tuning never makes it slower
  double best = per_default > 0 ? per_default : 1e300;
  int bb = c->block, bg = c->grid_per_sm, bk = c->graph_iters, bw = c->row_chunk;
  int tried = 0;
  for (int gi : graphs)
    for (int vw : widths)
      for (int bl : blocks)
        for (int g : gps) {
          if (g * bl > 2048) continue;  // the reduction grid stays resident
          c->graph_iters = gi;
          c->row_chunk = vw;
          c->block = bl;
          c->grid_per_sm = g;
          drop_graphs(c);
          double per = 0.0;
          if ((rc = measure(per))) return rc;
          ++tried;
          if (per > 0 && per < best) {
            best = per;
            bb = bl; bg = g; bk = gi; bw = vw;
          }
        }
  c->precision = precision;
  c->inner_max_iter = inner_keep;
  c->block = bb;
  c->grid_per_sm = bg;
  c->graph_iters = bk;
  c->row_chunk = bw;
  drop_graphs(c);
  rc = build_segments(c, c->seg_c0_caller, c->seg_c1_caller);
  if (rc) return rc;
  if (out) {
    out->block = bb;
    out->grid_per_sm = bg;
    out->graph_iters = bk;
    out->ms_per_iter = best;
    out->candidates = tried;
    out->vector_width = bw;
    out->ms_per_iter_before = per_default;
  }
  return SOLV_GPU_OK;
}

// ---- learned preconditioner: solve, inference, training ---------------------------
int solv_gpu_fcg(solv_gpu_ctx* c, double reduc, int n_iter, double* phi, double* res0,
                 double* res0_n, int not_r0, solv_gpu_stats* st) {
  return solve_host(c, 2, 0, reduc, n_iter, 1, phi, res0, res0_n, not_r0, st);
}
int solv_gpu_fcg_dev(solv_gpu_ctx* c, double reduc, int n_iter, double* phi, double* res0,
                     double* res0_n, int not_r0, solv_gpu_stats* st) {
  return solve_common(c, 2, 0, reduc, n_iter, 1, phi, res0, res0_n, not_r0, st);
}

int solv_gpu_mg_aggregate(int n, const long long* ptr, const int* adj, const float* w,
                          int passes, int* agg, int* n_agg) {
  if (n <= 0 || !ptr || !adj || !w || !agg || !n_agg || passes < 1 || passes > 8)
    return SOLV_GPU_BAD_INPUT;
  mg::Graph g;
  g.n = n;
  g.ptr.assign(ptr, ptr + n + 1);
  if (g.ptr[0] != 0) return SOLV_GPU_BAD_INPUT;
  for (int i = 0; i < n; ++i)
    if (g.ptr[i + 1] < g.ptr[i]) return SOLV_GPU_BAD_INPUT;
  const long long m = g.ptr[n];
  g.adj.assign(adj, adj + m);
  g.w.assign(w, w + m);
  for (long long k = 0; k < m; ++k)
    if (g.adj[k] < 0 || g.adj[k] >= n) return SOLV_GPU_BAD_INPUT;
  std::vector<int> a;
  *n_agg = mg::aggregate(g, passes, a);
  std::copy(a.begin(), a.end(), agg);
  return SOLV_GPU_OK;
}

int solv_gpu_mg_aggregates(solv_gpu_ctx* c, int level, int* agg, int n, int* n_coarse) {
  if (!c || !agg || !n_coarse) return set_err(c, SOLV_GPU_BAD_INPUT, "mg aggregates: null pointer");
  if (!c->has_matrix) return set_err(c, SOLV_GPU_NO_MATRIX, "no matrix set");
  CUDA_TRY(c, cudaSetDevice(c->dev));
  int rc = mg_setup(c);
  if (rc) return rc;
  if (level < 1 || level > (int)c->mg.size())
    return set_err(c, SOLV_GPU_BAD_INPUT, "mg aggregates: no such level");
  const int nf = level == 1 ? c->N : c->mg[level - 2]->n;
  if (n != nf) return set_err(c, SOLV_GPU_BAD_INPUT, "mg aggregates: n must be the finer level's size");
  std::vector<int> a(nf);
  CUDA_TRY(c, cudaMemcpyAsync(a.data(), c->mg[level - 1]->agg_of.p, nf * sizeof(int),
                              cudaMemcpyDeviceToHost, c->stream));
  std::vector<int> o2n;
  if (level == 1) {
    o2n.resize(nf);
    CUDA_TRY(c, cudaMemcpyAsync(o2n.data(), c->old_of_new.p, nf * sizeof(int),
                                cudaMemcpyDeviceToHost, c->stream));
  }
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  for (int i = 0; i < nf; ++i) agg[level == 1 ? o2n[i] : i] = a[i];
  *n_coarse = c->mg[level - 1]->n;
  return SOLV_GPU_OK;
}

int solv_gpu_gnn_n_params(void) { return gnn::N_PARAM; }

int solv_gpu_gnn_set_params(solv_gpu_ctx* c, const float* p, int n) {
  if (!c || !p || n != gnn::N_PARAM) return set_err(c, SOLV_GPU_BAD_INPUT, "gnn: expected N_PARAM floats");
  CUDA_TRY(c, cudaSetDevice(c->dev));
  const size_t b = gnn::N_PARAM_PAD * sizeof(float);
  CUDA_TRY(c, c->g_param.ensure(b));
  CUDA_TRY(c, c->g_grad.ensure(b));
  CUDA_TRY(c, c->g_m.ensure(b));
  CUDA_TRY(c, c->g_v.ensure(b));
  CUDA_TRY(c, cudaMemsetAsync(c->g_param.p, 0, b, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(c->g_param.p, p, n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemsetAsync(c->g_grad.p, 0, b, c->stream));
  CUDA_TRY(c, cudaMemsetAsync(c->g_m.p, 0, b, c->stream));
  CUDA_TRY(c, cudaMemsetAsync(c->g_v.p, 0, b, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  c->g_has_params = true;
  c->g_wcat_valid = false;
  c->g_adam_t = 0;
  return SOLV_GPU_OK;
}

int solv_gpu_gnn_get_params(solv_gpu_ctx* c, float* p, int n) {
  if (!c || !p || n != gnn::N_PARAM || !c->g_has_params)
    return set_err(c, SOLV_GPU_BAD_INPUT, "gnn: no parameters / bad size");
  CUDA_TRY(c, cudaMemcpy(p, c->g_param.p, n * sizeof(float), cudaMemcpyDeviceToHost));
  return SOLV_GPU_OK;
}

int solv_gpu_gnn_get_grad(solv_gpu_ctx* c, float* g, int n) {
  if (!c || !g || n != gnn::N_PARAM || !c->g_has_params)
    return set_err(c, SOLV_GPU_BAD_INPUT, "gnn: no parameters / bad size");
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  CUDA_TRY(c, cudaMemcpy(g, c->g_grad.p, n * sizeof(float), cudaMemcpyDeviceToHost));
  return SOLV_GPU_OK;
}

int solv_gpu_gnn_zero_grad(solv_gpu_ctx* c) {
  if (!c || !c->g_has_params) return set_err(c, SOLV_GPU_BAD_INPUT, "gnn: no parameters");
  CUDA_TRY(c, cudaMemsetAsync(c->g_grad.p, 0, gnn::N_PARAM_PAD * sizeof(float), c->stream));
  return SOLV_GPU_OK;
}

// Training buffers: 15 FP32 arrays of N x 32, 14 of N, 2 per slot.
enum { TB_H0 = 0, TB_AGG0 = 4, TB_PRE0 = 7, TB_DHA = 11, TB_DHB = 12, TB_DHS = 13, TB_DAGG = 14,
       TB_R0 = 15, TB_U0, TB_PA, TB_S, TB_HE, TB_RS, TB_US, TB_ZS, TB_GS, TB_Y, TB_DT, TB_DS,
       TB_ES, TB_Q, TB_EPRE, TB_GE, TB_COUNT };
static int gnn_train_buffers(solv_gpu_ctx* c, float** B) {
  const size_t nh = (size_t)c->N * gnn::H, n1 = (size_t)c->N, ns = (size_t)c->n_slots;
  CUDA_TRY(c, c->g_train.ensure((15 * nh + 14 * n1 + 2 * ns) * sizeof(float)));
  float* p = c->g_train.as<float>();
  for (int k = 0; k < 15; ++k, p += nh) B[k] = p;
  for (int k = TB_R0; k <= TB_Q; ++k, p += n1) B[k] = p;
  B[TB_EPRE] = p;
  B[TB_GE] = p + ns;
  return SOLV_GPU_OK;
}

// r (caller layout, device) -> internal FP32 and its scale gs in lane 0
static int gnn_load_residual(solv_gpu_ctx* c, const double* r_dev, float* rf) {
  const int N = c->N;
  sg::k_phi_in<float><<<grid_for(c, N), c->block, 0, c->stream>>>(N, 1, c->old_of_new.as<int>(),
                                                                  r_dev, rf);
  Lane L{};
  L.active = 1;
  CUDA_TRY(c, cudaMemcpyAsync(c->lanes.p, &L, sizeof(Lane), cudaMemcpyHostToDevice, c->stream));
  sg::k_fcg_scale<float><<<c->seg.total_blk, c->block, 0, c->stream>>>(
      segmap(c), rf, c->g_rsd.as<float>(), c->part.as<double>(), c->lanes.as<Lane>());
  CUDA_TRY(c, cudaGetLastError());
  return SOLV_GPU_OK;
}

__global__ void k_gnn_scaled_u(int n, const float* __restrict__ rsd, const float* __restrict__ r,
                               const Lane* __restrict__ lanes, float* __restrict__ u) {
  const double s = lanes[0].gs > 0 ? lanes[0].gs : 1.0;
  const float inv = (float)(1.0 / s);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    u[i] = r[i] * rsd[i] * inv;
}
__global__ void k_gnn_mul(int n, const float* __restrict__ a, const float* __restrict__ b,
                          float* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = a[i] * b[i];
}

// Training-path forward from the feature residual r0 (FP32 CUDA cores, BF16
// rounding as inference): activations, heads (s in the scaled space), faces.
static int gnn_train_forward(solv_gpu_ctx* c, const double* r0_dev, float** B) {
  int rc = gnn_load_residual(c, r0_dev, B[TB_R0]);
  if (rc) return rc;
  const int N = c->N;
  gnn::Feat F = gnn_feat(c);
  const float* P = c->g_param.as<float>();
  const int gw = gnn_grid_warps(c, (long long)N * 32);
  gnn::k_gnn_enc<float><<<gw, 256, 0, c->stream>>>(N, F, B[TB_R0], P, c->lanes.as<Lane>(),
                                                    c->g_h0.as<__nv_bfloat16>(), B[TB_U0]);
  gnn::k_gnn_enc_train<<<gw, 256, 0, c->stream>>>(N, F, B[TB_U0], P, B[TB_H0], B[TB_PRE0]);
  const int lb = std::max(1, std::min((N + 7) / 8, c->n_sm * 8));
  for (int l = 0; l < gnn::NL; ++l)
    gnn::k_gnn_layer_train<<<lb, 256, 0, c->stream>>>(
        N, rows<float>(c), F, B[TB_H0 + l], B[TB_AGG0 + l], B[TB_PRE0 + 1 + l], B[TB_H0 + 1 + l],
        P + gnn::P_LAYER + l * gnn::LAYER_SZ);
  gnn::k_gnn_heads<float><<<grid_for(c, N), 256, 0, c->stream>>>(N, B[TB_H0 + 3], P, nullptr, B[TB_PA],
                                                     B[TB_S], B[TB_HE]);
  gnn::k_gnn_edges<<<grid_for(c, N), c->block, 0, c->stream>>>(N, rows<float>(c), F, B[TB_HE], P,
                                                               B[TB_EPRE], B[TB_GE]);
  CUDA_TRY(c, cudaGetLastError());
  return SOLV_GPU_OK;
}

// z = M^-1 r with the preconditioner built from r0 (caller layout, device):
// path 0 = inference kernels (BF16, tensor cores), 1 = training kernels.
int solv_gpu_gnn_forward_dev(solv_gpu_ctx* c, const double* r0_dev, const double* r_dev,
                             double* z_dev, int path) {
  if (!c) return SOLV_GPU_BAD_INPUT;
  if (!c->has_matrix) return set_err(c, SOLV_GPU_NO_MATRIX, "no matrix set");
  if (!r0_dev || !r_dev || !z_dev) return set_err(c, SOLV_GPU_BAD_INPUT, "gnn forward: null pointer");
  CUDA_TRY(c, cudaSetDevice(c->dev));
  int rc = gnn_prepare(c);
  if (rc) return rc;
  float* B[TB_COUNT];
  if ((rc = gnn_train_buffers(c, B))) return rc;
  const int N = c->N;
  const int* o2n = c->old_of_new.as<int>();
  const float *q, *ge;
  if (path == 0) {
    if ((rc = gnn_load_residual(c, r0_dev, B[TB_R0]))) return rc;
    gnn_build<float>(c, B[TB_R0]);
    q = c->g_q.as<float>();
    ge = c->g_ge.as<float>();
  } else {
    if ((rc = gnn_train_forward(c, r0_dev, B))) return rc;
    k_gnn_mul<<<grid_for(c, N), c->block, 0, c->stream>>>(N, B[TB_S], c->g_rsd.as<float>(),
                                                           B[TB_Q]);
    q = B[TB_Q];
    ge = B[TB_GE];
  }
  sg::k_phi_in<float><<<grid_for(c, N), c->block, 0, c->stream>>>(N, 1, o2n, r_dev, B[TB_RS]);
  gnn::k_gnn_apply<float><<<grid_for(c, N), c->block, 0, c->stream>>>(N, rows<float>(c), ge, q,
                                                                      B[TB_RS], B[TB_ZS], nullptr);
  sg::k_phi_out<float><<<grid_for(c, N), c->block, 0, c->stream>>>(N, 1, o2n, B[TB_ZS], z_dev);
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  CUDA_TRY(c, cudaGetLastError());
  return SOLV_GPU_OK;
}

// One sample of the loss through the V-cycle (the smoother of level 0 is the
// training-path network: s in B[TB_S] as q = s rsd in B[TB_Q], faces in
// B[TB_GE]): forward V-cycle, loss L = -(z.b)^2/(z.Az) and its gradient,
// then the adjoint of the V-cycle, which gives the gradient with respect to
// each of the two smoother applications; the scaled-space backward kernels
// turn those into the gradients of s and of the face pre-activations.
static int mg_train_sample(solv_gpu_ctx* c, float** B) {
  const int N = c->N;
  const int G = grid_for(c, N), Bk = c->block;
  cudaStream_t s = c->stream;
  Rows<float> R0 = rows<float>(c);
  gnn::Feat F = gnn_feat(c);
  const float w = (float)c->mg_omega, a = (float)c->mg_alpha;
  const float* rsd = c->g_rsd.as<float>();
  const float* q = B[TB_Q];
  // smoother 2 trains the diagonal alone: the face weights stay zero
  const float* ge = c->mg_smoother == 2 ? c->g_zero.as<float>() : B[TB_GE];
  float* T = c->mg_train.as<float>();
  float *b = T, *z = T + N, *az = T + 2 * (size_t)N, *gz = T + 3 * (size_t)N;
  float *uh = T + 4 * (size_t)N, *gh = T + 5 * (size_t)N, *tmp = T + 6 * (size_t)N;
  float* gx = T + 7 * (size_t)N;
  float* x0 = c->mg_x0.as<float>();
  float* t0 = c->mg_t0.as<float>();
  MgLevel& L1 = *c->mg[0];
  double* sums = c->g_jsum.as<double>() + 1;
  auto back = [&](const float* u, const float* g) {
    gnn::k_gnn_apply_back1<<<G, Bk, 0, s>>>(N, B[TB_S], u, g, B[TB_Y], B[TB_DT]);
    gnn::k_gnn_apply_back2<<<G, Bk, 0, s>>>(N, R0, F, ge, B[TB_EPRE], u, g, B[TB_Y], B[TB_DT],
                                            B[TB_DS], B[TB_ES]);
  };
  mg::k_mg_normalise<<<G, Bk, 0, s>>>(N, B[TB_RS], c->lanes.as<Lane>(), b);
  mg_vcycle<float>(c, b, z, 1, q, ge, x0, t0, nullptr);  // t0 = b - A x before post-smoothing
  CUDA_TRY(c, cudaMemsetAsync(sums, 0, 2 * sizeof(double), s));
  mg::k_mg_loss_sums<<<G, 256, 0, s>>>(N, R0, z, b, az, sums);
  mg::k_mg_loss_grad<<<G, Bk, 0, s>>>(N, az, b, sums, gz, c->g_jsum.as<double>());
  // post-smoother z = x + w K t: its input t0, its output gradient gz
  mg::k_mg_scaled_pair<<<G, Bk, 0, s>>>(N, rsd, w, t0, gz, uh, gh);
  back(uh, gh);
  // adjoint to x (before post-smoothing): gx = gz - A (w K gz)
  mg::k_mg_net<false, float><<<G, Bk, 0, s>>>(N, R0, ge, q, w, gz, nullptr, tmp, nullptr);
  mg::k_mg_resid<<<G, Bk, 0, s>>>(N, R0, gz, tmp, gx, nullptr);
  // through the coarse correction x += a P C P^T (b - A x): gx -= A (a P C P^T gx)
  mg::k_mg_restrict<<<grid_for(c, L1.n), Bk, 0, s>>>(L1.n, L1.agg_ptr.as<int>(),
                                                     L1.agg_cells.as<int>(), gx, L1.b.as<float>(),
                                                     nullptr);
  mg_coarse_cycle(c, nullptr);
  CUDA_TRY(c, cudaMemsetAsync(tmp, 0, (size_t)N * sizeof(float), s));
  mg::k_mg_prolong<<<G, Bk, 0, s>>>(N, L1.agg_of.as<int>(), a, L1.y.as<float>(), tmp, nullptr);
  mg::k_mg_resid<<<G, Bk, 0, s>>>(N, R0, gx, tmp, az, nullptr);  // az = adjoint at x = w K b
  // pre-smoother x = w K b: its input b, its output gradient az
  mg::k_mg_scaled_pair<<<G, Bk, 0, s>>>(N, rsd, w, b, az, uh, gh);
  back(uh, gh);
  CUDA_TRY(c, cudaGetLastError());
  return SOLV_GPU_OK;
}

// Forward + backward of the energy loss J = 1/2 z.Â z - z.u, z = K u, for
// the preconditioner built from r0 and the n_samples residual samples r_k
// (each n_cell long, caller layout, consecutive; each normalised to unit
// mean magnitude).  Gradients add up in the FP32 accumulator (zeroed first
// unless accumulate); loss = mean over samples of J / n_cell.
int solv_gpu_gnn_grad_dev(solv_gpu_ctx* c, const double* r0_dev, const double* samples_dev,
                          int n_samples, double* loss, int accumulate) {
  if (!c) return SOLV_GPU_BAD_INPUT;
  if (!c->has_matrix) return set_err(c, SOLV_GPU_NO_MATRIX, "no matrix set");
  if (!r0_dev || !samples_dev || n_samples < 1)
    return set_err(c, SOLV_GPU_BAD_INPUT, "gnn grad: bad arguments");
  CUDA_TRY(c, cudaSetDevice(c->dev));
  int rc = gnn_prepare(c);
  if (rc) return rc;
  float* B[TB_COUNT];
  if ((rc = gnn_train_buffers(c, B))) return rc;
  if (!accumulate) CUDA_TRY(c, cudaMemsetAsync(c->g_grad.p, 0, gnn::N_PARAM_PAD * sizeof(float), c->stream));
  if ((rc = gnn_train_forward(c, r0_dev, B))) return rc;
  const int N = c->N;
  gnn::Feat F = gnn_feat(c);
  const float* P = c->g_param.as<float>();
  float* G = c->g_grad.as<float>();
  const int* o2n = c->old_of_new.as<int>();
  CUDA_TRY(c, c->g_jsum.ensure(3 * sizeof(double)));
  CUDA_TRY(c, cudaMemsetAsync(c->g_jsum.p, 0, sizeof(double), c->stream));
  CUDA_TRY(c, cudaMemsetAsync(B[TB_DS], 0, N * sizeof(float), c->stream));
  CUDA_TRY(c, cudaMemsetAsync(B[TB_ES], 0, N * sizeof(float), c->stream));
  if (c->gnn_loss == 2) {  // through the V-cycle: hierarchy and smoother in the original space
    if (c->mg_smoother == 0)
      return set_err(c, SOLV_GPU_BAD_INPUT, "gnn grad: the multigrid loss needs the network "
                                            "as smoother (SOLV_OPT_MG_SMOOTHER 1 or 2)");
    if ((rc = mg_setup(c))) return rc;
    if (c->mg.empty())
      return set_err(c, SOLV_GPU_BAD_INPUT, "gnn grad: the multigrid loss needs a hierarchy "
                                            "(system too small, or coarsening stalled)");
    if (c->mg_smoother == 2) {
      CUDA_TRY(c, c->g_zero.ensure(std::max<long long>(c->n_slots, 1) * sizeof(float)));
      CUDA_TRY(c, cudaMemsetAsync(c->g_zero.p, 0, std::max<long long>(c->n_slots, 1) * sizeof(float),
                                  c->stream));
    }
    if ((rc = mg_values(c))) return rc;
    CUDA_TRY(c, c->mg_train.ensure((size_t)8 * N * sizeof(float)));
    k_gnn_mul<<<grid_for(c, N), c->block, 0, c->stream>>>(N, B[TB_S], c->g_rsd.as<float>(),
                                                           B[TB_Q]);
  }
  for (int k = 0; k < n_samples; ++k) {
    if ((rc = gnn_load_residual(c, samples_dev + (size_t)k * N, B[TB_RS]))) return rc;
    if (c->gnn_loss == 2) {
      if ((rc = mg_train_sample(c, B))) return rc;
      continue;
    }
    // gnn_load_residual permuted the sample in; normalise it
    k_gnn_scaled_u<<<grid_for(c, N), c->block, 0, c->stream>>>(N, c->g_rsd.as<float>(), B[TB_RS],
                                                              c->lanes.as<Lane>(), B[TB_US]);
    gnn::k_gnn_apply<float><<<grid_for(c, N), c->block, 0, c->stream>>>(
        N, rows<float>(c), B[TB_GE], B[TB_S], B[TB_US], B[TB_ZS], nullptr);
    if (c->gnn_loss == 0) {
      gnn::k_gnn_loss_grad<<<grid_for(c, N), 256, 0, c->stream>>>(
          N, rows<float>(c), F, B[TB_ZS], B[TB_US], B[TB_GS], c->g_jsum.as<double>());
    } else {  // scale-free: energy after the best step along z
      double* sums = c->g_jsum.as<double>() + 1;
      CUDA_TRY(c, cudaMemsetAsync(sums, 0, 2 * sizeof(double), c->stream));
      gnn::k_gnn_az_sums<<<grid_for(c, N), 256, 0, c->stream>>>(N, rows<float>(c), F, B[TB_ZS],
                                                                B[TB_US], B[TB_GS], sums);
      gnn::k_gnn_scalefree_grad<<<grid_for(c, N), 256, 0, c->stream>>>(
          N, B[TB_GS], B[TB_US], sums, B[TB_GS], c->g_jsum.as<double>());
    }
    gnn::k_gnn_apply_back1<<<grid_for(c, N), c->block, 0, c->stream>>>(N, B[TB_S], B[TB_US],
                                                                      B[TB_GS], B[TB_Y], B[TB_DT]);
    gnn::k_gnn_apply_back2<<<grid_for(c, N), c->block, 0, c->stream>>>(
        N, rows<float>(c), F, B[TB_GE], B[TB_EPRE], B[TB_US], B[TB_GS], B[TB_Y], B[TB_DT],
        B[TB_DS], B[TB_ES]);
  }
  (void)o2n;
  const int gw = gnn_grid_warps(c, (long long)N * 32);
  const float gsc = 1.0f / ((float)N * (float)n_samples);
  if (c->gnn_loss == 2 && c->mg_smoother == 2)  // the face weights are not used
    CUDA_TRY(c, cudaMemsetAsync(B[TB_ES], 0, N * sizeof(float), c->stream));
  gnn::k_gnn_heads_back<<<gw, 256, 0, c->stream>>>(N, B[TB_H0 + 3], B[TB_PA], B[TB_S], B[TB_DS],
                                                   B[TB_ES], gsc, P, B[TB_DHA], G);
  float* dcur = B[TB_DHA];
  const int lb = std::max(1, std::min((N + 7) / 8, c->n_sm * 8));
  for (int l = gnn::NL - 1; l >= 0; --l) {
    const float* L = P + gnn::P_LAYER + l * gnn::LAYER_SZ;
    gnn::k_gnn_layer_back1<<<lb, 256, 0, c->stream>>>(
        N, B[TB_H0 + l], B[TB_AGG0 + l], B[TB_PRE0 + 1 + l], dcur, L, B[TB_DHS], B[TB_DAGG],
        G + gnn::P_LAYER + l * gnn::LAYER_SZ);
    float* dnext = dcur == B[TB_DHA] ? B[TB_DHB] : B[TB_DHA];
    gnn::k_gnn_layer_back2<<<gw, 256, 0, c->stream>>>(N, rows<float>(c), F, B[TB_DHS], B[TB_DAGG],
                                                      dnext);
    dcur = dnext;
  }
  gnn::k_gnn_enc_back<<<gw, 256, 0, c->stream>>>(N, F, B[TB_U0], B[TB_PRE0], dcur, G);
  CUDA_TRY(c, cudaGetLastError());
  double j = 0;
  CUDA_TRY(c, cudaMemcpyAsync(&j, c->g_jsum.p, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (loss) *loss = j / N / n_samples;
  return SOLV_GPU_OK;
}

// Adam step on the accumulated gradient (times grad_scale), then zero it.
int solv_gpu_gnn_adam(solv_gpu_ctx* c, float lr, float grad_scale) {
  if (!c || !c->g_has_params) return set_err(c, SOLV_GPU_BAD_INPUT, "gnn: no parameters");
  CUDA_TRY(c, cudaSetDevice(c->dev));
  c->g_adam_t++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float bc1 = 1.0f - std::pow(b1, (float)c->g_adam_t);
  const float bc2 = 1.0f - std::pow(b2, (float)c->g_adam_t);
  gnn::k_adam<<<(gnn::N_PARAM + 255) / 256, 256, 0, c->stream>>>(
      gnn::N_PARAM, c->g_param.as<float>(), c->g_grad.as<float>(), c->g_m.as<float>(),
      c->g_v.as<float>(), lr, b1, b2, 1e-8f, bc1, bc2, grad_scale);
  CUDA_TRY(c, cudaMemsetAsync(c->g_grad.p, 0, gnn::N_PARAM_PAD * sizeof(float), c->stream));
  CUDA_TRY(c, cudaGetLastError());
  c->g_wcat_valid = false;
  return SOLV_GPU_OK;
}

// ---- batches of independent systems ------------------------------------------
int solv_gpu_matrix_set_batch(solv_gpu_ctx* c, int n_sys, const int* cell_ptr, int n_face,
                              const int* ip, const int* in, const double* p, const double* n,
                              const double* pl) {
  if (!c) return SOLV_GPU_BAD_INPUT;
  if (n_sys < 1 || !cell_ptr || !p || !n || !pl)
    return set_err(c, SOLV_GPU_BAD_INPUT, "matrix_set_batch: bad arguments");
  CUDA_TRY(c, cudaSetDevice(c->dev));
  c->has_matrix = false;
  int rc = matrix_structure(c, cell_ptr[n_sys], n_face, ip, in, n_sys, cell_ptr);
  if (rc) return rc;
  return solv_gpu_matrix_values(c, p, n, pl);
}

int solv_gpu_n_systems(const solv_gpu_ctx* c) { return c && c->has_matrix ? c->n_seg : 0; }

int solv_gpu_cg_batch(solv_gpu_ctx* c, int imat, double reduc, int n_iter, int n_vc, double* phi,
                      double* res0, double* res0_n, int not_r0, int* iters, double* ratio,
                      solv_gpu_stats* st) {
  return solve_host(c, 0, imat, reduc, n_iter, n_vc, phi, res0, res0_n, not_r0, st, iters, ratio, true);
}
int solv_gpu_bicg_batch(solv_gpu_ctx* c, int imat, double reduc, int n_iter, int n_vc, double* phi,
                        double* res0, double* res0_n, int not_r0, int* iters, double* ratio,
                        solv_gpu_stats* st) {
  return solve_host(c, 1, imat, reduc, n_iter, n_vc, phi, res0, res0_n, not_r0, st, iters, ratio, true);
}
int solv_gpu_cg_batch_dev(solv_gpu_ctx* c, int imat, double reduc, int n_iter, int n_vc,
                          double* phi, double* res0, double* res0_n, int not_r0, int* iters,
                          double* ratio, solv_gpu_stats* st) {
  return solve_common(c, 0, imat, reduc, n_iter, n_vc, phi, res0, res0_n, not_r0, st, iters, ratio, true);
}
int solv_gpu_bicg_batch_dev(solv_gpu_ctx* c, int imat, double reduc, int n_iter, int n_vc,
                            double* phi, double* res0, double* res0_n, int not_r0, int* iters,
                            double* ratio, solv_gpu_stats* st) {
  return solve_common(c, 1, imat, reduc, n_iter, n_vc, phi, res0, res0_n, not_r0, st, iters, ratio, true);
}

// ---- Fortran bindings ----------------------------------------------------------
static solv_gpu_ctx* fctx(int64_t* h) { return h ? reinterpret_cast<solv_gpu_ctx*>(*h) : nullptr; }

void solv_gpu_create_(int64_t* h, int* device, int* status) {
  solv_gpu_ctx* c = nullptr;
  int rc = solv_gpu_create(&c, device ? *device : 0);
  if (h) *h = reinterpret_cast<int64_t>(c);
  if (status) *status = rc;
}
void solv_gpu_destroy_(int64_t* h, int* status) {
  int rc = solv_gpu_destroy(fctx(h));
  if (h) *h = 0;
  if (status) *status = rc;
}
void solv_gpu_matrix_set_(int64_t* h, int* n_cell, int* n_face, const int* ip, const int* in,
                          const double* p, const double* n, const double* pl, int* status) {
  int rc = (n_cell && n_face) ? solv_gpu_matrix_set(fctx(h), *n_cell, *n_face, ip, in, p, n, pl)
                              : SOLV_GPU_BAD_INPUT;
  if (status) *status = rc;
}
void solv_gpu_matrix_values_(int64_t* h, const double* p, const double* n, const double* pl,
                             int* status) {
  int rc = solv_gpu_matrix_values(fctx(h), p, n, pl);
  if (status) *status = rc;
}
void solv_gpu_res_(int64_t* h, int* n_vc, const double* phi, double* res0, double* res0_n,
                   int* not_r0, int* status) {
  int rc = (n_vc && not_r0) ? solv_gpu_res(fctx(h), *n_vc, phi, res0, res0_n, *not_r0)
                            : SOLV_GPU_BAD_INPUT;
  if (status) *status = rc;
}
void solv_gpu_precond_(int64_t* h, int* imat, double* cc, double* cr, int* status) {
  int rc = imat ? solv_gpu_precond(fctx(h), *imat, cc, cr) : SOLV_GPU_BAD_INPUT;
  if (status) *status = rc;
}
void solv_gpu_direct_(int64_t* h, int* imat, const double* cc, const double* cr, double* x,
                      const double* b, int* status) {
  int rc = imat ? solv_gpu_direct(fctx(h), *imat, cc, cr, x, b) : SOLV_GPU_BAD_INPUT;
  if (status) *status = rc;
}
void solv_gpu_cg_(int64_t* h, int* imat, double* reduc, int* n_iter, int* n_vc, double* phi,
                  double* res0, double* res0_n, int* not_r0, int* status) {
  int rc = (imat && reduc && n_iter && n_vc && not_r0)
               ? solv_gpu_cg(fctx(h), *imat, *reduc, *n_iter, *n_vc, phi, res0, res0_n, *not_r0, nullptr)
               : SOLV_GPU_BAD_INPUT;
  if (status) *status = rc;
}
void solv_gpu_bicg_(int64_t* h, int* imat, double* reduc, int* n_iter, int* n_vc, double* phi,
                    double* res0, double* res0_n, int* not_r0, int* status) {
  int rc = (imat && reduc && n_iter && n_vc && not_r0)
               ? solv_gpu_bicg(fctx(h), *imat, *reduc, *n_iter, *n_vc, phi, res0, res0_n, *not_r0, nullptr)
               : SOLV_GPU_BAD_INPUT;
  if (status) *status = rc;
}

}  // extern "C"

namespace {
int solve_dispatch(solv_gpu_ctx* c, int solver, int imat, double reduc, int n_iter, int V,
                   double* phi_dev, double* res0_dev, double* res0_n, int not_r0,
                   solv_gpu_stats* st, int* oi, double* orat) {
  if (solver == 2) {  // flexible CG with the learned preconditioner, FP32 inner
    if (V != 1 || c->n_seg != 1)
      return set_err(c, SOLV_GPU_BAD_INPUT, "learned preconditioner: one system, n_vc = 1");
    return solve_mixed_reliable<1>(c, 2, 0, reduc, n_iter, phi_dev, res0_dev, res0_n, not_r0, st, oi, orat);
  }
  if (c->precision == 1 && solver == 0) {
    switch (V) {
      case 1: return solve_mixed_reliable<1>(c, 0, imat, reduc, n_iter, phi_dev, res0_dev, res0_n, not_r0, st, oi, orat);
      case 2: return solve_mixed_reliable<2>(c, 0, imat, reduc, n_iter, phi_dev, res0_dev, res0_n, not_r0, st, oi, orat);
      case 3: return solve_mixed_reliable<3>(c, 0, imat, reduc, n_iter, phi_dev, res0_dev, res0_n, not_r0, st, oi, orat);
      case 4: return solve_mixed_reliable<4>(c, 0, imat, reduc, n_iter, phi_dev, res0_dev, res0_n, not_r0, st, oi, orat);
    }
    return set_err(c, SOLV_GPU_BAD_INPUT, "n_vc must be 1..4");
  }
  if (c->precision == 1) {
    switch (V) {
      case 1: return solve_mixed<1>(c, solver, imat, reduc, n_iter, phi_dev, res0_dev, res0_n, not_r0, st, oi, orat);
      case 2: return solve_mixed<2>(c, solver, imat, reduc, n_iter, phi_dev, res0_dev, res0_n, not_r0, st, oi, orat);
      case 3: return solve_mixed<3>(c, solver, imat, reduc, n_iter, phi_dev, res0_dev, res0_n, not_r0, st, oi, orat);
      case 4: return solve_mixed<4>(c, solver, imat, reduc, n_iter, phi_dev, res0_dev, res0_n, not_r0, st, oi, orat);
    }
    return set_err(c, SOLV_GPU_BAD_INPUT, "n_vc must be 1..4");
  }
  switch (V) {
    case 1: return solve_fp64<1>(c, solver, imat, reduc, n_iter, phi_dev, res0_dev, res0_n, not_r0, st, oi, orat);
    case 2: return solve_fp64<2>(c, solver, imat, reduc, n_iter, phi_dev, res0_dev, res0_n, not_r0, st, oi, orat);
    case 3: return solve_fp64<3>(c, solver, imat, reduc, n_iter, phi_dev, res0_dev, res0_n, not_r0, st, oi, orat);
    case 4: return solve_fp64<4>(c, solver, imat, reduc, n_iter, phi_dev, res0_dev, res0_n, not_r0, st, oi, orat);
  }
  return set_err(c, SOLV_GPU_BAD_INPUT, "n_vc must be 1..4");
}
}  // namespace
