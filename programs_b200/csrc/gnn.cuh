// gnn.cuh -- learned preconditioner: a message-passing network over the
// face graph of the pressure matrix, applied to the residual inside
// flexible CG.
//
// Scaled system: D = diag(A), Â = D^-1/2 A D^-1/2 (unit diagonal), edge
// weight w_ij = -Â_ij.  Per application, with u_i = r_i / (sqrt(d_i) s),
// s = sum_i |r_i|/sqrt(d_i) / N (scale of the residual):
//   h0_i   = relu(W_in x_i),        x_i = [u_i, rowsum_i/d_i, deg_i/6, 1]
//   agg_i  = sum_j w_ij h^l_j                       (gather over the row)
//   h^{l+1}_i = h^l_i + relu(W_s h^l_i + W_n agg_i + b^l),  l = 0, 1, 2
//   out_i  = c u_i + w_out . h3_i
//   z_i    = s out_i / sqrt(d_i)
// so z scales with r, and with the network's correction zeroed
// (w_out = 0, c = 1) z is the Jacobi step D^-1 r.  Width 32, 3 layers.
//
// Inference: weights and hidden states in BF16, the per-cell MLP of each
// layer ([h | agg] (64) x W (64x32)) on the tensor cores with FP32
// accumulate (mma.sync m16n8k16, 16 cells per warp).
// Training: FP32 CUDA-core kernels that round weights and stored hidden
// states to BF16 exactly where inference does, save the activations, and
// back-propagate the energy loss J = 1/2 out^T Â out - out^T u (its
// minimiser is out = Â^-1 u, i.e. z = A^-1 r); gradients are accumulated
// in FP32 and applied by Adam.
#pragma once
#include <cuda_bf16.h>

#include "kernels.cuh"

namespace gnn {

constexpr int H = 32;  // width
constexpr int NF = 4;  // input features
constexpr int NL = 3;  // message-passing layers
// parameter vector (FP32 master copy)
constexpr int P_WIN = 0;                       // [H][NF]
constexpr int P_LAYER = H * NF;                // per layer: Ws[H][H], Wn[H][H], b[H]
constexpr int LAYER_SZ = 2 * H * H + H;
constexpr int P_WOUT = P_LAYER + NL * LAYER_SZ;  // [H]
constexpr int P_C = P_WOUT + H;                  // scalar skip weight
constexpr int N_PARAM = P_C + 1;
constexpr int N_PARAM_PAD = (N_PARAM + 7) & ~7;

// Per-matrix features, internal cell order.
struct Feat {
  const float* __restrict__ rsd;   // 1/sqrt(d_i)
  const float* __restrict__ frs;   // sum_j a_ij / d_i (off-diagonal row sum ratio)
  const float* __restrict__ fdeg;  // interior neighbours / 6
  const float* __restrict__ gw;    // w_ij per sliced-ELL slot
};

__device__ __forceinline__ float bf(float x) { return __bfloat162float(__float2bfloat16(x)); }

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

// ---- inference ---------------------------------------------------------------
// Encoder: one warp per cell, lane = channel.  u from r (any precision).
template <typename T>
__global__ void k_gnn_enc(int n, Feat F, const T* __restrict__ r, const float* __restrict__ P,
                          const sg::Lane* __restrict__ lanes, __nv_bfloat16* __restrict__ h0,
                          float* __restrict__ u_out, const int* __restrict__ n_active) {
  if (n_active && *n_active == 0) return;
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

// One message-passing layer on the tensor cores.  Block = 4 warps, each
// warp 16 cells: gather [h | agg] rows into shared memory (lane =
// channel), then C[16x32] = A[16x64] B[64x32] with 4 k-steps x 4 n-tiles of
// m16n8k16, then bias, relu, residual, store BF16.
constexpr int TC_CELLS = 16;
constexpr int TC_WARPS = 4;
__global__ void __launch_bounds__(TC_WARPS * 32)
k_gnn_layer_tc(int n, sg::Rows<float> R, Feat F, const __nv_bfloat16* __restrict__ hin,
               __nv_bfloat16* __restrict__ hout, const __nv_bfloat16* __restrict__ wcat,
               const float* __restrict__ bias, const int* __restrict__ n_active) {
  if (n_active && *n_active == 0) return;
  __shared__ __nv_bfloat16 sB[2 * H][H + 8];
  __shared__ __nv_bfloat16 sA[TC_WARPS][TC_CELLS][2 * H + 8];
  __shared__ float sbias[H];
  for (int t = threadIdx.x; t < 2 * H * H; t += blockDim.x) sB[t / H][t % H] = wcat[t];
  if (threadIdx.x < H) sbias[threadIdx.x] = bf(bias[threadIdx.x]);
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, tg = lane & 3;
  const int tiles = (n + TC_CELLS - 1) / TC_CELLS;
  for (int tile = blockIdx.x * TC_WARPS + w; tile < tiles; tile += gridDim.x * TC_WARPS) {
    const int c0 = tile * TC_CELLS;
    for (int cc = 0; cc < TC_CELLS; ++cc) {
      const int i = c0 + cc;
      __nv_bfloat16 hv = __float2bfloat16(0.0f), av = hv;
      if (i < n) {
        hv = hin[(size_t)i * H + lane];
        sg::RowIt<float> it(R, i);
        float agg = 0.0f;
        for (int k = 0; k < it.w; ++k) {
          const int e = it.base + k * sg::kWarp;
          const int j = R.col[e];
          if (j >= 0) agg += F.gw[e] * __bfloat162float(hin[(size_t)j * H + lane]);
        }
        av = __float2bfloat16(agg);
      }
      sA[w][cc][lane] = hv;
      sA[w][cc][H + lane] = av;
    }
    __syncwarp();
    float acc[4][4];
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[nt][q] = 0.0f;
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      const int k0 = ks * 16;
      const uint32_t a0 = pack_bf16(sA[w][g][k0 + 2 * tg], sA[w][g][k0 + 2 * tg + 1]);
      const uint32_t a1 = pack_bf16(sA[w][g + 8][k0 + 2 * tg], sA[w][g + 8][k0 + 2 * tg + 1]);
      const uint32_t a2 = pack_bf16(sA[w][g][k0 + 2 * tg + 8], sA[w][g][k0 + 2 * tg + 9]);
      const uint32_t a3 = pack_bf16(sA[w][g + 8][k0 + 2 * tg + 8], sA[w][g + 8][k0 + 2 * tg + 9]);
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int n0 = nt * 8;
        const uint32_t b0 = pack_bf16(sB[k0 + 2 * tg][n0 + g], sB[k0 + 2 * tg + 1][n0 + g]);
        const uint32_t b1 = pack_bf16(sB[k0 + 2 * tg + 8][n0 + g], sB[k0 + 2 * tg + 9][n0 + g]);
        mma_bf16(acc[nt], a0, a1, a2, a3, b0, b1);
      }
    }
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int row = g + (q >> 1) * 8, col = nt * 8 + 2 * tg + (q & 1);
        const int i = c0 + row;
        if (i < n) {
          const float pre = acc[nt][q] + sbias[col];
          const float hold = __bfloat162float(sA[w][row][col]);
          hout[(size_t)i * H + col] = __float2bfloat16(hold + fmaxf(pre, 0.0f));
        }
      }
    }
    __syncwarp();
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

// Decoder (training and inference share it): out = c u + w_out . h3; one
// warp per cell.  Training passes float h3; inference BF16.
template <typename HT>
__global__ void k_gnn_dec_out(int n, const HT* __restrict__ h3, const float* __restrict__ u,
                              const float* __restrict__ P, float* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const float wo = bf(P[P_WOUT + lane]), c = bf(P[P_C]);
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    float v = wo * (float)h3[(size_t)i * H + lane];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) out[i] = c * u[i] + v;
  }
}

// Inference decoder: out as above, then z_i = s out_i / sqrt(d_i).
template <typename T>
__global__ void k_gnn_dec_z(int n, Feat F, const __nv_bfloat16* __restrict__ h3,
                            const float* __restrict__ u, const float* __restrict__ P,
                            const sg::Lane* __restrict__ lanes, T* __restrict__ z,
                            const int* __restrict__ n_active) {
  if (n_active && *n_active == 0) return;
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const float wo = bf(P[P_WOUT + lane]), c = bf(P[P_C]);
  const double scale = lanes[0].gs > 0 ? lanes[0].gs : 1.0;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    float v = wo * __bfloat162float(h3[(size_t)i * H + lane]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) z[i] = (T)((double)(c * u[i] + v) * scale * F.rsd[i]);
  }
}

// Energy loss pieces: g = Â out - u (= dJ/dout) and J = 1/2 out.Â out - out.u
// (block partials, summed on the host side by the caller's reduction).
__global__ void k_gnn_loss_grad(int n, sg::Rows<float> R, Feat F, const float* __restrict__ out,
                                const float* __restrict__ u, float* __restrict__ g,
                                double* __restrict__ jsum) {
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    sg::RowIt<float> it(R, i);
    float aout = out[i];  // unit diagonal
    for (int k = 0; k < it.w; ++k) {
      const int e = it.base + k * sg::kWarp;
      const int j = R.col[e];
      if (j >= 0) aout -= F.gw[e] * out[j];
    }
    g[i] = aout - u[i];
    acc += 0.5 * (double)out[i] * aout - (double)out[i] * u[i];
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

// Decoder backward: dout (= g * scale) -> dW_out, dc, dh3.
__global__ void k_gnn_dec_back(int n, const float* __restrict__ h3, const float* __restrict__ u,
                               const float* __restrict__ dout, float gsc,
                               const float* __restrict__ P, float* __restrict__ dh3,
                               float* __restrict__ G) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const float wo = bf(P[P_WOUT + lane]);
  float gw = 0.0f, gc = 0.0f;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    const float d = dout[i] * gsc;
    gw += d * h3[(size_t)i * H + lane];
    if (lane == 0) gc += d * u[i];
    dh3[(size_t)i * H + lane] = d * wo;
  }
  atomicAdd(&G[P_WOUT + lane], gw);
  if (lane == 0) atomicAdd(&G[P_C], gc);
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
  const float g = G[t] * gscale;
  m[t] = b1 * m[t] + (1.0f - b1) * g;
  v[t] = b2 * v[t] + (1.0f - b2) * g * g;
  const float mh = m[t] / bc1, vh = v[t] / bc2;
  P[t] -= lr * mh / (sqrtf(vh) + eps);
}

}  // namespace gnn
