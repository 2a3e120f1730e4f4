// noalloc.cu -- solv_res for callers that cannot allocate device memory.
//
// Some host codes run where cudaMalloc is off limits: inside a memory pool
// another runtime owns, or under a no-allocation policy in a long-running
// service.  They hold the matrix
// (ng, pl) and the vectors in device memory they already own and need the
// residual r = b - A phi with its L1 norms (spray-simulation/solv_res.f90)
// without a context, a workspace or any allocation.
//
// solv_gpu_res_noalloc reads the face list and vectors in place and keeps
// its only scratch -- the per-block partial sums of the L1 reduction, a
// completion ticket and a bad-index counter -- in one file-scope
// __device__ array of fixed size (NaScratch below, about 19 KB), which every
// GPU that loads this library holds until the process exits.  Host code
// cannot pass that array's name to a kernel (it is a host-side stand-in,
// not a device address), so the first call on each device, with that device
// current, looks its address up with cudaGetSymbolAddress and caches it;
// make that first call before any stream capture.  All calls on a device
// share the one array: the ticket and counter are cleared at the start of
// every call, and calls that overlap on the GPU (different streams, no
// ordering between them) race on it.  Face indices are checked on the GPU
// before res0 is touched; a bad one leaves res0 and res0_n as they were.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "../../include/solv_gpu.h"

namespace {

constexpr int kNaBlocks = 592;  // 4 blocks per SM on 148 SMs
constexpr int kNaThreads = 256;
constexpr int kNaMaxVc = SOLV_GPU_MAX_VC;
constexpr int kNaMaxDevices = 64;

struct NaScratch {
  double part[kNaBlocks * kNaMaxVc];  // block partial L1 sums
  unsigned int ticket;                // blocks done (last one combines)
  int bad;                            // faces with an out-of-range index
};

static __device__ __align__(256) NaScratch g_na_scratch;

std::mutex g_na_mutex;
NaScratch* g_na_ptr[kNaMaxDevices] = {nullptr};

// Face indices checked before anything is written: a face whose ip or in
// lies outside 1..n (in = 0 marks a boundary face) counts in S->bad, and
// the kernels below leave res0 and res0_n alone when the count is not zero.
__global__ void k_na_check(int n, int nf, const int* __restrict__ ip, const int* __restrict__ in,
                           NaScratch* __restrict__ S) {
  int bad = 0;
  for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < nf;
       f += (long long)gridDim.x * blockDim.x) {
    const int a = ip[f], b = in[f];
    bad += (a < 1 || a > n || b < 0 || b > n);
  }
  if (bad) atomicAdd(&S->bad, bad);
}

// r_i -= pl_i phi_i (column-major r, cell-major phi)
__global__ void k_na_cells(int n, int nv, const double* __restrict__ pl,
                           const double* __restrict__ phi, double* __restrict__ r,
                           const NaScratch* __restrict__ S) {
  if (S->bad) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    for (int v = 0; v < nv; ++v)
      r[(size_t)v * n + i] -= pl[i] * phi[(size_t)i * nv + v];
}

// face loop of solv_res.f90:16-23; both updates of a face are atomic adds
__global__ void k_na_faces(int n, int nf, int nv, const int* __restrict__ ip,
                           const int* __restrict__ in, const double* __restrict__ p,
                           const double* __restrict__ nn, const double* __restrict__ phi,
                           double* __restrict__ r, const NaScratch* __restrict__ S) {
  if (S->bad) return;
  for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < nf;
       f += (long long)gridDim.x * blockDim.x) {
    if (in[f] == 0) continue;  // boundary face
    const int a = ip[f] - 1, b = in[f] - 1;
    for (int v = 0; v < nv; ++v) {
      atomicAdd(&r[(size_t)v * n + a], -p[f] * phi[(size_t)b * nv + v]);
      atomicAdd(&r[(size_t)v * n + b], -nn[f] * phi[(size_t)a * nv + v]);
    }
  }
}

// res0_n[v] = sum_i |r(i,v)|: fixed grid, partials in the static scratch,
// the last block to finish combines them in block order (deterministic).
__global__ void __launch_bounds__(kNaThreads)
k_na_l1(int n, int nv, const double* __restrict__ r, double* __restrict__ out,
        NaScratch* __restrict__ S) {
  __shared__ double sh[kNaMaxVc][kNaThreads / 32];
  __shared__ bool last;
  if (S->bad) return;
  double acc[kNaMaxVc] = {0.0, 0.0, 0.0, 0.0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    for (int v = 0; v < nv; ++v) acc[v] += fabs(r[(size_t)v * n + i]);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  for (int v = 0; v < kNaMaxVc; ++v) {
    double x = acc[v];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (l == 0) sh[v][w] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int v = 0; v < kNaMaxVc; ++v) {
      double x = 0.0;
      for (int k = 0; k < kNaThreads / 32; ++k) x += sh[v][k];
      S->part[blockIdx.x * kNaMaxVc + v] = x;
    }
    __threadfence();
    last = atomicAdd(&S->ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last || threadIdx.x >= 32) return;
  __threadfence();
  for (int v = 0; v < nv; ++v) {
    double x = 0.0;
    for (int b = l; b < (int)gridDim.x; b += 32) x += __ldcg(&S->part[b * kNaMaxVc + v]);
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (l == 0) out[v] = x;
  }
  if (l == 0) S->ticket = 0u;
}

// Device address of the static scratch for the current device (looked up
// once per device, under a lock).
int na_scratch(NaScratch** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNaMaxDevices)
    return SOLV_GPU_DEVICE_ERROR;
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (!g_na_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_na_scratch) != cudaSuccess || !p) return SOLV_GPU_DEVICE_ERROR;
    g_na_ptr[dev] = static_cast<NaScratch*>(p);
  }
  *out = g_na_ptr[dev];
  return SOLV_GPU_OK;
}

}  // namespace

extern "C" int solv_gpu_res_noalloc(int n_cell, int n_face, const int* ip, const int* in,
                                    const double* p, const double* n, const double* pl,
                                    int n_vc, const double* phi, double* res0,
                                    double* res0_n, int not_r0, void* stream) {
  if (n_cell <= 0 || n_face < 0 || n_vc < 1 || !ip || !in || !p || !n || !pl || !phi || !res0 ||
      !res0_n)
    return SOLV_GPU_BAD_INPUT;
  if (n_vc > kNaMaxVc) return SOLV_GPU_TOO_LARGE;  // the scratch holds 4 components
  NaScratch* S = nullptr;
  int rc = na_scratch(&S);
  if (rc) return rc;
  // a launch error left over from the caller's earlier work is not this
  // call's: clear it so that only these launches are checked below
  (void)cudaGetLastError();
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(&S->ticket, 0, sizeof(unsigned int) + sizeof(int), st) != cudaSuccess)
    return SOLV_GPU_DEVICE_ERROR;
  const int gc = (int)std::min<long long>(((long long)n_cell + kNaThreads - 1) / kNaThreads, 4096);
  const int gf = (int)std::min<long long>(((long long)n_face + kNaThreads - 1) / kNaThreads, 4096);
  if (!not_r0 && n_face > 0) k_na_check<<<gf, kNaThreads, 0, st>>>(n_cell, n_face, ip, in, S);
  if (!not_r0) {
    k_na_cells<<<gc, kNaThreads, 0, st>>>(n_cell, n_vc, pl, phi, res0, S);
    if (n_face > 0)
      k_na_faces<<<gf, kNaThreads, 0, st>>>(n_cell, n_face, n_vc, ip, in, p, n, phi, res0, S);
  }
  k_na_l1<<<kNaBlocks, kNaThreads, 0, st>>>(n_cell, n_vc, res0, res0_n, S);
  int bad = 0;
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(&bad, &S->bad, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return SOLV_GPU_DEVICE_ERROR;
  return bad ? SOLV_GPU_BAD_INPUT : SOLV_GPU_OK;
}
