// gnn.cuh -- learned preconditioner: a message-passing network over the
// face graph of the (symmetric) pressure matrix that builds, once per solve,
// a symmetric positive definite preconditioner applied in flexible CG.
//
// Scaled system: D = diag(A), Â = D^-1/2 A D^-1/2 (unit diagonal), edge
// weight w_ij = -Â_ij (w_ij = w_ji).  Network (width 32, 3 layers), inputs
// per cell x_i = [u0_i, rowsum_i/d_i, deg_i/6, 1] with u0 the initial
// residual scaled by D^-1/2 and by its mean magnitude:
//   h0_i      = relu(W_in x_i)
//   agg_i     = sum_j w_ij h^l_j                          (gather over the row)
//   h^{l+1}_i = h^l_i + relu(W_s h^l_i + W_n agg_i + b^l),  l = 0, 1, 2
// Heads (per cell, then per face):
//   s_i   = sqrt(softplus(w_a . h3_i + b_a) / softplus(0)) (diagonal scale > 0)
//   e_ij  = gamma tanh((w_e . h3_i + w_e . h3_j)/2 + b_e)  (symmetric in i, j)
// Preconditioner, linear in the residual:
//   M^-1 = D^-1/2 S (I + E) S D^-1/2,  S = diag(s),  E_ij = e_ij w_ij
// E is symmetric and, since sum_j w_ij <= 1 on these M-matrices and
// gamma < 1, I + E is diagonally dominant: M^-1 is symmetric positive
// definite for any weights, so CG keeps its optimality.  With w_a = w_e = 0,
// b_a = b_e = 0 it is exactly the Jacobi step D^-1.
// Applying it costs one gather over the rows per Krylov iteration:
//   z_i = q_i (q_i r_i + sum_j gE_ij q_j r_j),  q = S D^-1/2 r,  gE = E.
//
// Inference: weights and hidden states in BF16, the per-cell MLP of each
// layer ([h | agg] (64) x W (64x32)) on the tensor cores with FP32
// accumulate (mma.sync m16n8k16, 16 cells per warp).
// Training: FP32 CUDA-core kernels that round weights and stored hidden
// states to BF16 where inference does; the loss is the energy of the
// preconditioned step in the scaled space, J = 1/2 z.Â z - z.u with z = K u
// (K = S (I+E) S), minimised by K u = Â^-1 u, averaged over residual
// samples u of the same system.
#pragma once
#include <cuda_bf16.h>

#include <type_traits>

#include "kernels.cuh"

namespace gnn {

constexpr int H = 32;  // width
constexpr int NF = 4;  // input features
constexpr int NL = 3;  // message-passing layers
// parameter vector (FP32 master copy)
constexpr int P_WIN = 0;                         // [H][NF]
constexpr int P_LAYER = H * NF;                  // per layer: Ws[H][H], Wn[H][H], b[H]
constexpr int LAYER_SZ = 2 * H * H + H;
constexpr int P_WA = P_LAYER + NL * LAYER_SZ;    // [H] diagonal-scale head
constexpr int P_BA = P_WA + H;                   // scalar
constexpr int P_WE = P_BA + 1;                   // [H] face head
constexpr int P_BE = P_WE + H;                   // scalar
constexpr int N_PARAM = P_BE + 1;
constexpr int N_PARAM_PAD = (N_PARAM + 7) & ~7;
constexpr float kGamma = 0.95f;

// Per-matrix features, internal cell order.
struct Feat {
  const float* __restrict__ rsd;   // 1/sqrt(d_i)
  const float* __restrict__ frs;   // sum_j a_ij / d_i (off-diagonal row sum ratio)
  const float* __restrict__ fdeg;  // interior neighbours / 6
  const float* __restrict__ gw;    // w_ij per sliced-ELL slot
};

__device__ __forceinline__ float bf(float x) { return __bfloat162float(__float2bfloat16(x)); }
__device__ __forceinline__ float softplus(float x) { return x > 20.f ? x : log1pf(expf(x)); }
__device__ __forceinline__ float sigmoid(float x) { return 1.0f / (1.0f + expf(-x)); }

// ---- features ------------------------------------------------------------------
__global__ void k_gnn_features(int n, sg::Rows<double> R, float* __restrict__ rsd,
                               float* __restrict__ frs, float* __restrict__ fdeg,
                               float* __restrict__ gw) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    sg::RowIt<double> it(R, i);
    const double d = R.diag[i];
    const double ri = d > 0 ? 1.0 / sqrt(d) : 0.0;
    double rs = 0.0;
    int deg = 0;
    for (int k = 0; k < it.w; ++k) {
      const int e = it.base + k * sg::kWarp;
      const int j = R.col[e];
      if (j >= 0) {
        const double dj = R.diag[j];
        const double rj = dj > 0 ? 1.0 / sqrt(dj) : 0.0;
        gw[e] = (float)(-R.val[e] * ri * rj);
        rs += R.val[e];
        ++deg;
      } else {
        gw[e] = 0.0f;
      }
    }
    rsd[i] = (float)ri;
    frs[i] = d > 0 ? (float)(rs / d) : 0.0f;
    fdeg[i] = deg / 6.0f;
  }
}

// Pack layer l's [Ws | Wn] as the B operand (K = 64 rows, N = 32 cols),
// BF16: wcat[k][j] = Ws[j][k] (k < 32), Wn[j][k-32] (k >= 32).
__global__ void k_gnn_pack(const float* __restrict__ P, __nv_bfloat16* __restrict__ wcat) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= NL * 2 * H * H) return;
  const int l = t / (2 * H * H), r = t % (2 * H * H);
  const int k = r / H, j = r % H;
  const float* L = P + P_LAYER + l * LAYER_SZ;
  const float w = k < H ? L[j * H + k] : L[H * H + j * H + (k - H)];
  wcat[t] = __float2bfloat16(w);
}

// ---- network ------------------------------------------------------------------
// Encoder: one warp per cell, lane = channel; u = r rsd / gs (gs in lane 0).
template <typename T>
__global__ void k_gnn_enc(int n, Feat F, const T* __restrict__ r, const float* __restrict__ P,
                          const sg::Lane* __restrict__ lanes, __nv_bfloat16* __restrict__ h0,
                          float* __restrict__ u_out) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const double scale = lanes[0].gs > 0 ? lanes[0].gs : 1.0;  // sum |r| rsd / N
  const float inv_s = (float)(1.0 / scale);
  const float w0 = bf(P[P_WIN + lane * NF + 0]), w1 = bf(P[P_WIN + lane * NF + 1]);
  const float w2 = bf(P[P_WIN + lane * NF + 2]), w3 = bf(P[P_WIN + lane * NF + 3]);
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    const float u = (float)r[i] * F.rsd[i] * inv_s;
    const float v = w0 * u + w1 * F.frs[i] + w2 * F.fdeg[i] + w3;
    h0[(size_t)i * H + lane] = __float2bfloat16(fmaxf(v, 0.0f));
    if (lane == 0) u_out[i] = u;
  }
}

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  __nv_bfloat162 v;
  v.x = lo;
  v.y = hi;
  return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Four 8x8 BF16 matrices from shared memory into the mma fragment layout
// (lane l gives the address of row l & 15 of matrix l >> 4's column block);
// TRANS transposes each 8x8 matrix on the way (B stored k-major).
template <bool TRANS>
__device__ __forceinline__ void ldmatrix_x4(const __nv_bfloat16* p, uint32_t& r0, uint32_t& r1,
                                            uint32_t& r2, uint32_t& r3) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  if constexpr (TRANS)
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(a));
  else
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(a));
}

// One message-passing layer on the tensor cores.  Block = 4 warps, each
// warp 16 cells: gather [h | agg] rows into shared memory (lane =
// channel), then C[16x32] = A[16x64] B[64x32] with 4 k-steps x 4 n-tiles of
// m16n8k16, then bias, relu, residual; the BF16 result goes back into the
// warp's shared tile and out as whole 64-byte rows.
constexpr int TC_CELLS = 16;
constexpr int TC_WARPS = 4;
constexpr int TC_CHUNK = 4;  // neighbour rows loaded at once per lane
__global__ void __launch_bounds__(TC_WARPS * 32)
k_gnn_layer_tc(int n, sg::Rows<float> R, Feat F, const __nv_bfloat16* __restrict__ hin,
               __nv_bfloat16* __restrict__ hout, const __nv_bfloat16* __restrict__ wcat,
               const float* __restrict__ bias) {
  __shared__ __align__(16) __nv_bfloat16 sB[2 * H][H + 8];
  __shared__ __align__(16) __nv_bfloat16 sA[TC_WARPS][TC_CELLS][2 * H + 8];
  __shared__ float sbias[H];
  for (int t = threadIdx.x; t < 2 * H * H; t += blockDim.x) sB[t / H][t % H] = wcat[t];
  if (threadIdx.x < H) sbias[threadIdx.x] = bf(bias[threadIdx.x]);
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, tg = lane & 3;
  const int tiles = (n + TC_CELLS - 1) / TC_CELLS;
  for (int tile = blockIdx.x * TC_WARPS + w; tile < tiles; tile += gridDim.x * TC_WARPS) {
    const int c0 = tile * TC_CELLS;
    // gather: four lanes per cell row (8 channels each, one 16-byte load per
    // row), 8 cells of the tile at a time, TC_CHUNK neighbour rows in flight
    // per lane; per channel the neighbours add up in row order, as in the
    // training kernels
    const int sub = lane >> 2, cb = (lane & 3) * 8;
    for (int cc0 = 0; cc0 < TC_CELLS; cc0 += 8) {
      const int cc = cc0 + sub;
      const int i = c0 + cc;
      uint4 hv = make_uint4(0u, 0u, 0u, 0u);
      float af[8];
#pragma unroll
      for (int t = 0; t < 8; ++t) af[t] = 0.0f;
      if (i < n) {
        hv = *reinterpret_cast<const uint4*>(hin + (size_t)i * H + cb);
        sg::RowIt<float> it(R, i);
        for (int k0 = 0; k0 < it.w; k0 += TC_CHUNK) {
          int j[TC_CHUNK];
          float wg[TC_CHUNK];
          uint4 v[TC_CHUNK];
#pragma unroll
          for (int u = 0; u < TC_CHUNK; ++u) {
            j[u] = -1;
            wg[u] = 0.0f;
            if (k0 + u < it.w) {
              const int e = it.base + (k0 + u) * sg::kWarp;
              j[u] = __ldg(&R.col[e]);
              wg[u] = __ldg(&F.gw[e]);
            }
          }
#pragma unroll
          for (int u = 0; u < TC_CHUNK; ++u)
            v[u] = j[u] >= 0 ? __ldg(reinterpret_cast<const uint4*>(hin + (size_t)j[u] * H + cb))
                             : make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
          for (int u = 0; u < TC_CHUNK; ++u) {
            if (j[u] < 0) continue;
            const __nv_bfloat162* p2 = reinterpret_cast<const __nv_bfloat162*>(&v[u]);
#pragma unroll
            for (int t = 0; t < 4; ++t) {
              const float2 f = __bfloat1622float2(p2[t]);
              af[2 * t] += wg[u] * f.x;
              af[2 * t + 1] += wg[u] * f.y;
            }
          }
        }
      }
      uint4 av;
      __nv_bfloat162* a2 = reinterpret_cast<__nv_bfloat162*>(&av);
#pragma unroll
      for (int t = 0; t < 4; ++t) a2[t] = __floats2bfloat162_rn(af[2 * t], af[2 * t + 1]);
      *reinterpret_cast<uint4*>(&sA[w][cc][cb]) = hv;
      *reinterpret_cast<uint4*>(&sA[w][cc][H + cb]) = av;
    }
    __syncwarp();
    float acc[4][4];
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[nt][q] = 0.0f;
    // fragments by ldmatrix: A rows (lane & 15), k block (lane >> 4) of the
    // tile; B k rows (lane & 15) of two n tiles (lane >> 4), transposed
    const int lr = lane & 15, lc = (lane >> 4) * 8;
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      const int k0 = ks * 16;
      uint32_t a0, a1, a2, a3;
      ldmatrix_x4<false>(&sA[w][lr][k0 + lc], a0, a1, a2, a3);
#pragma unroll
      for (int nt = 0; nt < 4; nt += 2) {
        uint32_t b0, b1, b2, b3;  // (b0, b1) of tile nt, (b2, b3) of tile nt + 1
        ldmatrix_x4<true>(&sB[k0 + lr][nt * 8 + lc], b0, b1, b2, b3);
        mma_bf16(acc[nt], a0, a1, a2, a3, b0, b1);
        mma_bf16(acc[nt + 1], a0, a1, a2, a3, b2, b3);
      }
    }
    __syncwarp();  // every lane has read the tile: the result may overwrite h
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int row = g + (q >> 1) * 8, col = nt * 8 + 2 * tg + (q & 1);
        const float pre = acc[nt][q] + sbias[col];
        const float hold = __bfloat162float(sA[w][row][col]);
        sA[w][row][col] = __float2bfloat16(hold + fmaxf(pre, 0.0f));
      }
    }
    __syncwarp();
    // 16 rows x 64 bytes: two 16-byte stores a lane
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      const int idx = t * 32 + lane, row = idx >> 2, part = (idx & 3) * 8;
      const int i = c0 + row;
      if (i < n)
        *reinterpret_cast<uint4*>(hout + (size_t)i * H + part) =
            *reinterpret_cast<const uint4*>(&sA[w][row][part]);
    }
    __syncwarp();
  }
}

// Heads, per cell (one warp per cell): pa = w_a.h3 + b_a, s = sqrt(softplus(pa)),
// he = w_e.h3; q = s * qscale_i (qscale = rsd for the preconditioner, NULL = 1).
template <typename HT>
__global__ void k_gnn_heads(int n, const HT* __restrict__ h3, const float* __restrict__ P,
                            const float* __restrict__ qscale, float* __restrict__ pa_out,
                            float* __restrict__ s_out, float* __restrict__ he_out) {
  // one thread per cell; the 32 hidden channels of a cell are one
  // contiguous row (64 bytes in BF16: four 16-byte loads)
  __shared__ float swa[H], swe[H];
  if (threadIdx.x < H) {
    swa[threadIdx.x] = bf(P[P_WA + threadIdx.x]);
    swe[threadIdx.x] = bf(P[P_WE + threadIdx.x]);
  }
  __syncthreads();
  const float ba = bf(P[P_BA]);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float a = 0.0f, e = 0.0f;
    if constexpr (std::is_same<HT, __nv_bfloat16>::value) {
      const uint4* row = reinterpret_cast<const uint4*>(h3 + (size_t)i * H);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const uint4 v = row[q];
        const __nv_bfloat162* p2 = reinterpret_cast<const __nv_bfloat162*>(&v);
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          const float2 f = __bfloat1622float2(p2[t]);
          const int c = q * 8 + 2 * t;
          a = fmaf(swa[c], f.x, a);
          a = fmaf(swa[c + 1], f.y, a);
          e = fmaf(swe[c], f.x, e);
          e = fmaf(swe[c + 1], f.y, e);
        }
      }
    } else {
#pragma unroll 8
      for (int c = 0; c < H; ++c) {
        const float h = (float)h3[(size_t)i * H + c];
        a = fmaf(swa[c], h, a);
        e = fmaf(swe[c], h, e);
      }
    }
    const float pa = a + ba;
    const float s = sqrtf(softplus(pa) / softplus(0.0f));  // exactly 1 untrained
    if (pa_out) pa_out[i] = pa;
    s_out[i] = qscale ? s * qscale[i] : s;
    he_out[i] = e;
  }
}

// Face weights per sliced-ELL slot: gE = gamma tanh((he_i + he_j)/2 + b_e) w_ij.
__global__ void k_gnn_edges(int n, sg::Rows<float> R, Feat F, const float* __restrict__ he,
                            const float* __restrict__ P, float* __restrict__ epre,
                            float* __restrict__ gE) {
  const float be = bf(P[P_BE]);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    sg::RowIt<float> it(R, i);
    const float hi = he[i];
    for (int k = 0; k < it.w; ++k) {
      const int e = it.base + k * sg::kWarp;
      const int j = R.col[e];
      float g = 0.0f;
      if (j >= 0) {
        const float pre = 0.5f * (hi + he[j]) + be;
        if (epre) epre[e] = pre;
        g = kGamma * tanhf(pre) * F.gw[e];
      }
      gE[e] = g;
    }
  }
}

// z = q (q r + E (q r)): the preconditioner application (one row gather).
template <typename T>
__global__ void k_gnn_apply(int n, sg::Rows<float> R, const float* __restrict__ gE,
                            const float* __restrict__ q, const T* __restrict__ r,
                            T* __restrict__ z, const int* __restrict__ n_active) {
  if (n_active && *n_active == 0) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    sg::RowIt<float> it(R, i);
    const float qi = q[i];
    float t = qi * (float)r[i];
    for (int k = 0; k < it.w; ++k) {
      const int e = it.base + k * sg::kWarp;
      const int j = R.col[e];
      if (j >= 0) t += gE[e] * q[j] * (float)r[j];
    }
    z[i] = (T)(qi * t);
  }
}

// ---- training (FP32 CUDA cores, BF16 rounding where inference rounds) ------------
// Encoder with saved pre-activations.  Thread per (cell, channel).
__global__ void k_gnn_enc_train(int n, Feat F, const float* __restrict__ u,
                                const float* __restrict__ P, float* __restrict__ h0,
                                float* __restrict__ pre0) {
  const long long tot = (long long)n * H;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / H), ch = (int)(t % H);
    const float* w = P + P_WIN + ch * NF;
    const float v = bf(w[0]) * u[i] + bf(w[1]) * F.frs[i] + bf(w[2]) * F.fdeg[i] + bf(w[3]);
    pre0[t] = v;
    h0[t] = bf(fmaxf(v, 0.0f));
  }
}

// One layer forward (training): agg (saved), pre (saved), h_out (BF16-rounded).
// Block = 8 cells x 32 channels.
__global__ void __launch_bounds__(256)
k_gnn_layer_train(int n, sg::Rows<float> R, Feat F, const float* __restrict__ hin,
                  float* __restrict__ agg_out, float* __restrict__ pre_out,
                  float* __restrict__ hout, const float* __restrict__ L) {
  __shared__ float sW[2 * H][H + 1];  // [k][j]
  __shared__ float sa[8][2 * H];
  __shared__ float sb[H];
  for (int t = threadIdx.x; t < 2 * H * H; t += blockDim.x) {
    const int k = t / H, j = t % H;
    sW[k][j] = bf(k < H ? L[j * H + k] : L[H * H + j * H + (k - H)]);
  }
  if (threadIdx.x < H) sb[threadIdx.x] = bf(L[2 * H * H + threadIdx.x]);
  __syncthreads();
  const int cl = threadIdx.x >> 5, ch = threadIdx.x & 31;
  for (int base = blockIdx.x * 8; base < n; base += gridDim.x * 8) {
    const int i = base + cl;
    if (i < n) {
      sg::RowIt<float> it(R, i);
      float agg = 0.0f;
      for (int k = 0; k < it.w; ++k) {
        const int e = it.base + k * sg::kWarp;
        const int j = R.col[e];
        if (j >= 0) agg += F.gw[e] * hin[(size_t)j * H + ch];
      }
      agg = bf(agg);
      agg_out[(size_t)i * H + ch] = agg;
      sa[cl][ch] = hin[(size_t)i * H + ch];
      sa[cl][H + ch] = agg;
    }
    __syncthreads();
    if (i < n) {
      float pre = sb[ch];
#pragma unroll 8
      for (int k = 0; k < 2 * H; ++k) pre += sW[k][ch] * sa[cl][k];
      pre_out[(size_t)i * H + ch] = pre;
      hout[(size_t)i * H + ch] = bf(sa[cl][ch] + fmaxf(pre, 0.0f));
    }
    __syncthreads();
  }
}

// Energy loss of one sample: g = Â z - u (= dJ/dz), J = 1/2 z.Â z - z.u.
__global__ void k_gnn_loss_grad(int n, sg::Rows<float> R, Feat F, const float* __restrict__ z,
                                const float* __restrict__ u, float* __restrict__ g,
                                double* __restrict__ jsum) {
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    sg::RowIt<float> it(R, i);
    float az = z[i];  // unit diagonal
    for (int k = 0; k < it.w; ++k) {
      const int e = it.base + k * sg::kWarp;
      const int j = R.col[e];
      if (j >= 0) az -= F.gw[e] * z[j];
    }
    g[i] = az - u[i];
    acc += 0.5 * (double)z[i] * az - (double)z[i] * u[i];
  }
  acc = sg::warp_sum(acc);
  __shared__ double sh[32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x + 31) / 32 ? sh[threadIdx.x] : 0.0;
    v = sg::warp_sum(v);
    if (threadIdx.x == 0) atomicAdd(jsum, v);
  }
}

// Scale-free variant of the loss: the energy after the best step along z,
// L = -(z.u)^2 / (z.Â z), whose gradient is 2 a (a Â z - u) with
// a = z.u / z.Â z -- CG does not see the scale of M^-1, and neither does L.
// Pass 1: Âz and the sums z.Âz, z.u; pass 2 (this kernel): g from them.
__global__ void k_gnn_az_sums(int n, sg::Rows<float> R, Feat F, const float* __restrict__ z,
                              const float* __restrict__ u, float* __restrict__ az_out,
                              double* __restrict__ sums) {
  double a0 = 0.0, a1 = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    sg::RowIt<float> it(R, i);
    float az = z[i];
    for (int k = 0; k < it.w; ++k) {
      const int e = it.base + k * sg::kWarp;
      const int j = R.col[e];
      if (j >= 0) az -= F.gw[e] * z[j];
    }
    az_out[i] = az;
    a0 += (double)z[i] * az;
    a1 += (double)z[i] * u[i];
  }
  a0 = sg::warp_sum(a0);
  a1 = sg::warp_sum(a1);
  __shared__ double sh[2][32];
  if ((threadIdx.x & 31) == 0) {
    sh[0][threadIdx.x >> 5] = a0;
    sh[1][threadIdx.x >> 5] = a1;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const bool in = threadIdx.x < (blockDim.x + 31) / 32;
    double v0 = in ? sh[0][threadIdx.x] : 0.0, v1 = in ? sh[1][threadIdx.x] : 0.0;
    v0 = sg::warp_sum(v0);
    v1 = sg::warp_sum(v1);
    if (threadIdx.x == 0) {
      atomicAdd(&sums[0], v0);
      atomicAdd(&sums[1], v1);
    }
  }
}
// g = 2 a (a Â z - u), a = z.u / z.Âz; adds L = -(z.u)^2/(z.Âz) to jsum
// (once, from thread 0 of block 0).
__global__ void k_gnn_scalefree_grad(int n, const float* __restrict__ az,
                                     const float* __restrict__ u, const double* __restrict__ sums,
                                     float* __restrict__ g, double* __restrict__ jsum) {
  const double zaz = sums[0] > 0.0 ? sums[0] : 1e-300, zu = sums[1];
  const double a = zu / zaz;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    g[i] = (float)(2.0 * a * (a * (double)az[i] - (double)u[i]));
  if (blockIdx.x == 0 && threadIdx.x == 0) *jsum += -zu * zu / zaz;
}

// Backward through z = S (I + E) S u for one sample (S = diag(s)):
//   y = s u, dt = s g, t = y + E y, dy = dt + E dt,
//   ds_i  += g_i t_i + dy_i u_i
//   esum_i += sum_j (dt_i y_j + dt_j y_i) gamma w_ij sech^2(pre_ij)
// (esum_i is the derivative w.r.t. the face pre-activations touching i).
__global__ void k_gnn_apply_back1(int n, const float* __restrict__ s, const float* __restrict__ u,
                                  const float* __restrict__ g, float* __restrict__ y,
                                  float* __restrict__ dt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    y[i] = s[i] * u[i];
    dt[i] = s[i] * g[i];
  }
}
__global__ void k_gnn_apply_back2(int n, sg::Rows<float> R, Feat F, const float* __restrict__ gE,
                                  const float* __restrict__ epre, const float* __restrict__ u,
                                  const float* __restrict__ g, const float* __restrict__ y,
                                  const float* __restrict__ dt, float* __restrict__ ds,
                                  float* __restrict__ esum) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    sg::RowIt<float> it(R, i);
    float t = y[i], edt = 0.0f, es = 0.0f;
    const float dti = dt[i], yi = y[i];
    for (int k = 0; k < it.w; ++k) {
      const int e = it.base + k * sg::kWarp;
      const int j = R.col[e];
      if (j >= 0) {
        t += gE[e] * y[j];
        edt += gE[e] * dt[j];
        const float th = tanhf(epre[e]);
        es += (dti * y[j] + dt[j] * yi) * kGamma * F.gw[e] * (1.0f - th * th);
      }
    }
    ds[i] += g[i] * t + (dti + edt) * u[i];
    esum[i] += es;
  }
}

// Heads backward (one warp per cell): from ds (w.r.t. s) and esum,
// dpa = ds sigmoid(pa) / (2 s), dhe = esum / 2, dh3 = dpa w_a + dhe w_e,
// and the head parameter gradients.  gsc scales everything (1/(N samples)).
__global__ void k_gnn_heads_back(int n, const float* __restrict__ h3, const float* __restrict__ pa,
                                 const float* __restrict__ s, const float* __restrict__ ds,
                                 const float* __restrict__ esum, float gsc,
                                 const float* __restrict__ P, float* __restrict__ dh3,
                                 float* __restrict__ G) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const float wa = bf(P[P_WA + lane]), we = bf(P[P_WE + lane]);
  float gwa = 0.f, gwe = 0.f, gba = 0.f, gbe = 0.f;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    const float dpa = ds[i] * gsc * sigmoid(pa[i]) / (2.0f * s[i] * softplus(0.0f));
    const float dhe = 0.5f * esum[i] * gsc;
    const float h = h3[(size_t)i * H + lane];
    dh3[(size_t)i * H + lane] = dpa * wa + dhe * we;
    gwa += dpa * h;
    gwe += dhe * h;
    if (lane == 0) {
      gba += dpa;
      gbe += dhe;  // d/d b_e = sum over faces = 1/2 sum_i esum_i
    }
  }
  atomicAdd(&G[P_WA + lane], gwa);
  atomicAdd(&G[P_WE + lane], gwe);
  if (lane == 0) {
    atomicAdd(&G[P_BA], gba);
    atomicAdd(&G[P_BE], gbe);
  }
}

// Layer backward, step 1 (per cell): dpre = dh_out * [pre > 0];
// dh_self = dh_out + Ws^T dpre; dagg = Wn^T dpre; dWs += dpre h^T,
// dWn += dpre agg^T, db += dpre.  Block = 8 cells x 32 channels.
__global__ void __launch_bounds__(256)
k_gnn_layer_back1(int n, const float* __restrict__ hin, const float* __restrict__ agg,
                  const float* __restrict__ pre, const float* __restrict__ dhout,
                  const float* __restrict__ L, float* __restrict__ dh_self,
                  float* __restrict__ dagg, float* __restrict__ GL) {
  __shared__ float sW[2 * H][H + 1];  // [k][j] = W[j][k]
  __shared__ float sd[8][H];          // dpre
  __shared__ float sx[8][2 * H];      // [h | agg]
  __shared__ float gacc[2 * H][H + 1];
  __shared__ float gb[H];
  for (int t = threadIdx.x; t < 2 * H * H; t += blockDim.x) {
    const int k = t / H, j = t % H;
    sW[k][j] = bf(k < H ? L[j * H + k] : L[H * H + j * H + (k - H)]);
    gacc[k][j] = 0.0f;
  }
  if (threadIdx.x < H) gb[threadIdx.x] = 0.0f;
  __syncthreads();
  const int cl = threadIdx.x >> 5, ch = threadIdx.x & 31;
  for (int base = blockIdx.x * 8; base < n; base += gridDim.x * 8) {
    const int i = base + cl;
    float dp = 0.0f, dho = 0.0f;
    if (i < n) {
      const size_t q = (size_t)i * H + ch;
      dho = dhout[q];
      dp = pre[q] > 0.0f ? dho : 0.0f;
      sx[cl][ch] = hin[q];
      sx[cl][H + ch] = agg[q];
    } else {
      sx[cl][ch] = 0.0f;
      sx[cl][H + ch] = 0.0f;
    }
    sd[cl][ch] = dp;
    __syncthreads();
    if (i < n) {
      float ds = dho, da = 0.0f;
#pragma unroll 8
      for (int j = 0; j < H; ++j) {
        const float dj = sd[cl][j];
        ds += sW[ch][j] * dj;       // Ws^T dpre : W[j][ch]
        da += sW[H + ch][j] * dj;   // Wn^T dpre
      }
      dh_self[(size_t)i * H + ch] = ds;
      dagg[(size_t)i * H + ch] = da;
    }
    // weight gradients: thread (cl, ch) owns inputs k = cl*4 .. cl*4+3 of
    // both halves (8 warps x 4 = the 32 inputs of h and of agg)
    for (int kk = 0; kk < 4; ++kk) {
      const int k = cl * 4 + kk;
      float s1 = 0.0f, s2 = 0.0f;
#pragma unroll
      for (int c2 = 0; c2 < 8; ++c2) {
        s1 += sd[c2][ch] * sx[c2][k];
        s2 += sd[c2][ch] * sx[c2][H + k];
      }
      gacc[k][ch] += s1;
      gacc[H + k][ch] += s2;
    }
    if (cl == 0) {
      float s = 0.0f;
#pragma unroll
      for (int c2 = 0; c2 < 8; ++c2) s += sd[c2][ch];
      gb[ch] += s;
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < 2 * H * H; t += blockDim.x) {
    const int k = t / H, j = t % H;
    // dWs[j][k] (k < 32) / dWn[j][k-32]
    const int off = k < H ? j * H + k : H * H + j * H + (k - H);
    atomicAdd(&GL[off], gacc[k][j]);
  }
  if (threadIdx.x < H) atomicAdd(&GL[2 * H * H + threadIdx.x], gb[threadIdx.x]);
}

// Layer backward, step 2 (gather, w symmetric): dh_in_i = dh_self_i + sum_j w_ij dagg_j.
__global__ void k_gnn_layer_back2(int n, sg::Rows<float> R, Feat F,
                                  const float* __restrict__ dh_self,
                                  const float* __restrict__ dagg, float* __restrict__ dhin) {
  const long long tot = (long long)n * H;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / H), ch = (int)(t % H);
    sg::RowIt<float> it(R, i);
    float v = dh_self[t];
    for (int k = 0; k < it.w; ++k) {
      const int e = it.base + k * sg::kWarp;
      const int j = R.col[e];
      if (j >= 0) v += F.gw[e] * dagg[(size_t)j * H + ch];
    }
    dhin[t] = v;
  }
}

// Encoder backward: dW_in += dpre0 x^T.
__global__ void k_gnn_enc_back(int n, Feat F, const float* __restrict__ u,
                               const float* __restrict__ pre0, const float* __restrict__ dh0,
                               float* __restrict__ G) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  float g0 = 0, g1 = 0, g2 = 0, g3 = 0;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    const size_t q = (size_t)i * H + lane;
    const float d = pre0[q] > 0.0f ? dh0[q] : 0.0f;
    g0 += d * u[i];
    g1 += d * F.frs[i];
    g2 += d * F.fdeg[i];
    g3 += d;
  }
  atomicAdd(&G[P_WIN + lane * NF + 0], g0);
  atomicAdd(&G[P_WIN + lane * NF + 1], g1);
  atomicAdd(&G[P_WIN + lane * NF + 2], g2);
  atomicAdd(&G[P_WIN + lane * NF + 3], g3);
}

// Adam (bias-corrected), FP32 master weights.
__global__ void k_adam(int np, float* __restrict__ P, const float* __restrict__ G,
                       float* __restrict__ m, float* __restrict__ v, float lr, float b1,
                       float b2, float eps, float bc1, float bc2, float gscale) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= np) return;
  // a non-finite gradient entry (a degenerate sample) is skipped: once in
  // the moments it would turn the parameter into NaN for good
  const float graw = G[t] * gscale;
  const float g = isfinite(graw) ? graw : 0.0f;
  m[t] = b1 * m[t] + (1.0f - b1) * g;
  v[t] = b2 * v[t] + (1.0f - b2) * g * g;
  const float mh = m[t] / bc1, vh = v[t] / bc2;
  P[t] -= lr * mh / (sqrtf(vh) + eps);
}

}  // namespace gnn
