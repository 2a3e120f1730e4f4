// fv_gpu.cu -- the SIMPLE outer-loop pieces on the GPU (include/fv_gpu.h).
//
// The reference assembles the momentum and pressure-correction matrices,
// the Green-Gauss gradients and the corrections in face loops over
// ng(:)%{ip,in} (cfd_setup.f90:178-431, 473-518, 604-646, 765-866).  A face
// loop scatters into both of its cells; on the GPU the face terms are
// computed one thread per face, and each cell then gathers its faces in
// ascending face order (a cell -> face list built once), which is the order
// the face loop adds them in -- so the sums, and every output, are bit-for-
// bit the host restatement's in fvmesh.cpp.  All double arithmetic below is
// written with explicit round-to-nearest operations (no fused multiply-add),
// as a compiler without FMA contraction evaluates the host code.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/fv_gpu.h"
#include "../../include/solv_gpu.h"

namespace {

__device__ __forceinline__ double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double da(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double ds(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dd(double a, double b) { return __ddiv_rn(a, b); }
// w a_N + (1 - w) a_P: linear interpolation to the face
__device__ __forceinline__ double lerp(double w, double an, double ap) {
  return da(dm(w, an), dm(ds(1.0, w), ap));
}

struct Geo {
  int n_cell, n_face;
  const int *ip, *in;          // 0-based, in = -1 on boundary faces
  const double *s, *nrm, *xf, *l, *w;
  const double *xc, *vol;
  const int *cf_ptr, *cf;      // faces of each cell, ascending
};

// std::min / std::max as the host evaluates them (ties and NaN included)
__device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }

// displacement from a cell centre xc to its auxiliary point on the face:
// (x_f - n ((x_f - x_c).n)) - x_c, the host's V3 operations in order
struct Dx {
  double x, y, z;
};
__device__ __forceinline__ double dot3(double ax, double ay, double az, double bx, double by,
                                       double bz) {
  return da(da(dm(ax, bx), dm(ay, by)), dm(az, bz));
}
__device__ __forceinline__ Dx aux_dx(const Geo& g, int f, int c) {
  const double* xf = g.xf + 3 * f;
  const double* nn = g.nrm + 3 * f;
  const double* xc = g.xc + 3 * c;
  const double t = dot3(ds(xf[0], xc[0]), ds(xf[1], xc[1]), ds(xf[2], xc[2]), nn[0], nn[1], nn[2]);
  return {ds(ds(xf[0], dm(nn[0], t)), xc[0]), ds(ds(xf[1], dm(nn[1], t)), xc[1]),
          ds(ds(xf[2], dm(nn[2], t)), xc[2])};
}


constexpr int kBlock = 256;
constexpr int kRedBlocks = 1024;

int grid(long long n) { return (int)std::max(1LL, std::min((n + kBlock - 1) / kBlock, 148LL * 16)); }

// d = rho (1/a_P)_f area V_f / l_pn (cfd_setup.f90:604-634)
__device__ __forceinline__ double pc_coef(const Geo& g, int f, int a, int b, const double* ap,
                                          double rho) {
  const double w = g.w[f];
  const double p_r = da(dd(w, da(ap[b], 1e-20)), dd(ds(1.0, w), da(ap[a], 1e-20)));
  const double v = lerp(w, g.vol[b], g.vol[a]);
  return dd(dm(dm(dm(rho, p_r), g.s[f]), v), g.l[f]);
}

// ---- momentum ---------------------------------------------------------------------
__global__ void k_fv_mom_faces(Geo g, const double* __restrict__ u, const double* __restrict__ flux,
                               double rho, double mu, double* __restrict__ p, double* __restrict__ n,
                               double* __restrict__ flux_out) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < g.n_face; f += gridDim.x * blockDim.x) {
    const int a = g.ip[f], b = g.in[f];
    const double d = dd(dm(mu, g.s[f]), g.l[f]);
    if (b >= 0) {
      double c;
      if (flux) {
        c = flux[f];
      } else {
        const double w = g.w[f];
        const double uf = lerp(w, u[3 * b], u[3 * a]);
        const double vf = lerp(w, u[3 * b + 1], u[3 * a + 1]);
        const double wf = lerp(w, u[3 * b + 2], u[3 * a + 2]);
        const double un = da(da(dm(uf, g.nrm[3 * f]), dm(vf, g.nrm[3 * f + 1])),
                             dm(wf, g.nrm[3 * f + 2]));
        c = dm(dm(rho, g.s[f]), un);
      }
      if (flux_out) flux_out[f] = c;
      const double mn = (0.0 < c) ? 0.0 : c;  // std::min(c, 0.0)
      const double mx = (c < 0.0) ? 0.0 : c;  // std::max(c, 0.0)
      p[f] = da(-d, mn);
      n[f] = ds(-d, mx);
    } else {
      if (flux_out) flux_out[f] = 0.0;
      p[f] = -d;
      n[f] = 0.0;
    }
  }
}

__global__ void k_fv_mom_cells(Geo g, const double* __restrict__ u, const double* __restrict__ p,
                               const double* __restrict__ n, double u_lid, double urf,
                               double* __restrict__ pl, double* __restrict__ rhs) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < g.n_cell; c += gridDim.x * blockDim.x) {
    double s = 0.0, rx = 0.0;
    for (int q = g.cf_ptr[c]; q < g.cf_ptr[c + 1]; ++q) {
      const int f = g.cf[q];
      if (g.in[f] < 0) {
        const double d = -p[f];
        s = da(s, d);
        // the moving lid: the y = 1 wall (outward normal +y)
        if (g.nrm[3 * f + 1] > 0.9 && g.xf[3 * f + 1] > 1.0 - 1e-9) rx = da(rx, dm(d, u_lid));
      } else if (g.ip[f] == c) {
        s = ds(s, p[f]);
      } else {
        s = ds(s, n[f]);
      }
    }
    s = dd(s, urf);
    pl[c] = s;
    if (rhs) {
      const double k = dm(ds(1.0, urf), s);
      rhs[3 * c] = da(rx, dm(k, u[3 * c]));
      rhs[3 * c + 1] = da(0.0, dm(k, u[3 * c + 1]));
      rhs[3 * c + 2] = da(0.0, dm(k, u[3 * c + 2]));
    }
  }
}

// ---- pressure correction ----------------------------------------------------------
__global__ void k_fv_pc_faces(Geo g, const double* __restrict__ ap, double rho, int pc,
                              double* __restrict__ dface, double* __restrict__ p,
                              double* __restrict__ n) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < g.n_face; f += gridDim.x * blockDim.x) {
    const int a = g.ip[f], b = g.in[f];
    double d = 0.0, off = 0.0;
    if (b >= 0) {
      d = pc_coef(g, f, a, b, ap, rho);
      if (a != pc && b != pc) off = -d;
    }
    dface[f] = d;
    p[f] = off;
    n[f] = off;
  }
}

__global__ void k_fv_pc_cells(Geo g, const double* __restrict__ dface, double* __restrict__ pl) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < g.n_cell; c += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int q = g.cf_ptr[c]; q < g.cf_ptr[c + 1]; ++q) {
      const int f = g.cf[q];
      if (g.in[f] >= 0) s = da(s, dface[f]);
    }
    pl[c] = s;
  }
}

// ---- Green-Gauss gradient -----------------------------------------------------------
__global__ void k_fv_gradient(Geo g, int nc, const double* __restrict__ phi,
                              double* __restrict__ grad) {
  const long long tot = (long long)g.n_cell * nc;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t / nc), k = (int)(t % nc);
    double gx = 0.0, gy = 0.0, gz = 0.0;
    for (int q = g.cf_ptr[c]; q < g.cf_ptr[c + 1]; ++q) {
      const int f = g.cf[q];
      const int a = g.ip[f], b = g.in[f];
      const double pa = phi[(size_t)a * nc + k];
      const double pf = b >= 0 ? lerp(g.w[f], phi[(size_t)b * nc + k], pa) : pa;
      const double ps = dm(pf, g.s[f]);
      const double tx = dm(ps, g.nrm[3 * f]), ty = dm(ps, g.nrm[3 * f + 1]),
                   tz = dm(ps, g.nrm[3 * f + 2]);
      if (a == c) {
        gx = da(gx, tx); gy = da(gy, ty); gz = da(gz, tz);
      } else {
        gx = ds(gx, tx); gy = ds(gy, ty); gz = ds(gz, tz);
      }
    }
    const double v = g.vol[c];
    double* o = grad + ((size_t)c * nc + k) * 3;
    o[0] = dd(gx, v);
    o[1] = dd(gy, v);
    o[2] = dd(gz, v);
  }
}

// ---- solv_grad in full: corrected Green-Gauss sweeps ---------------------------------
// One sweep of fvm_gradient_sweeps (cfd_setup.f90:765-866): the face value
// of each face (previous sweep's gradient g0 at the auxiliary points after
// the first sweep; walls by neu), its term ((phi_f s) n) / V added by each
// of the face's cells in ascending face order, 1/V (vr) formed once per
// cell.  bval[f*nc + k] are the wall values for neu = 0.
__device__ __forceinline__ double sweep_face_value(const Geo& g, int f, int nc, int k,
                                                   const double* __restrict__ phi,
                                                   const double* __restrict__ bval, int neu,
                                                   const double* __restrict__ g0) {
  const int a = g.ip[f], b = g.in[f];
  const double pa = phi[(size_t)a * nc + k];
  const double* ga0 = g0 ? g0 + ((size_t)a * nc + k) * 3 : nullptr;
  if (b >= 0) {
    const double pb = phi[(size_t)b * nc + k];
    if (g0) {
      const double* gb0 = g0 + ((size_t)b * nc + k) * 3;
      const Dx xa = aux_dx(g, f, a), xb = aux_dx(g, f, b);
      const double pp = da(pa, dot3(ga0[0], ga0[1], ga0[2], xa.x, xa.y, xa.z));
      const double pn = da(pb, dot3(gb0[0], gb0[1], gb0[2], xb.x, xb.y, xb.z));
      return lerp(g.w[f], pn, pp);
    }
    return lerp(g.w[f], pb, pa);
  }
  if (neu > 0) {
    double pf = pa;
    if (g0 && neu == 2) {
      const double* xf = g.xf + 3 * f;
      const double* xc = g.xc + 3 * a;
      pf = da(pf, dot3(ga0[0], ga0[1], ga0[2], ds(xf[0], xc[0]), ds(xf[1], xc[1]),
                       ds(xf[2], xc[2])));
    }
    return pf;
  }
  return bval[(size_t)f * nc + k];
}

__global__ void k_fv_grad_sweep(Geo g, int nc, const double* __restrict__ phi,
                                const double* __restrict__ bval, int neu,
                                const double* __restrict__ vr, const double* __restrict__ g0,
                                double* __restrict__ grad) {
  const long long tot = (long long)g.n_cell * nc;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t / nc), k = (int)(t % nc);
    double gx = 0.0, gy = 0.0, gz = 0.0;
    const double v = vr[c];
    for (int q = g.cf_ptr[c]; q < g.cf_ptr[c + 1]; ++q) {
      const int f = g.cf[q];
      const double ps = dm(sweep_face_value(g, f, nc, k, phi, bval, neu, g0), g.s[f]);
      const double* nn = g.nrm + 3 * f;
      const double tx = dm(dm(ps, nn[0]), v), ty = dm(dm(ps, nn[1]), v),
                   tz = dm(dm(ps, nn[2]), v);
      if (g.ip[f] == c) {
        gx = da(gx, tx); gy = da(gy, ty); gz = da(gz, tz);
      } else {
        gx = ds(gx, tx); gy = ds(gy, ty); gz = ds(gz, tz);
      }
    }
    double* o = grad + ((size_t)c * nc + k) * 3;
    o[0] = gx;
    o[1] = gy;
    o[2] = gz;
  }
}

__global__ void k_fv_recip(int n, const double* __restrict__ vol, double* __restrict__ vr) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    vr[c] = dd(1.0, vol[c]);  // cfd_grid.f90:546
}

// ---- explicit momentum terms: fvm_momentum_deferred ------------------------------------
// Per interior face and component (cfd_setup.f90:185-272, 306-328):
// cor = c_bl c (phi_up - phi_f) + d ((phi_N' - phi_P') - (phi_N - phi_P)),
// the face value by `scheme` (0 central, 1 min-mod, 2 van Leer, 3 superbee
// on the auxiliary-point values); then each cell adds +cor (owner) or
// -cor (neighbour) of its faces in ascending face order.
__global__ void k_fv_deferred_faces(Geo g, int nc, const double* __restrict__ phi,
                                    const double* __restrict__ grad,
                                    const double* __restrict__ flux, double mu, double c_bl,
                                    int scheme, double* __restrict__ cor) {
  const long long tot = (long long)g.n_face * nc;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(t / nc), k = (int)(t % nc);
    const int a = g.ip[f], b = g.in[f];
    if (b < 0) {
      cor[t] = 0.0;
      continue;
    }
    const double w = g.w[f];
    const Dx xa = aux_dx(g, f, a), xb = aux_dx(g, f, b);
    const double c = flux[f], d = dd(dm(mu, g.s[f]), g.l[f]);
    const double pa = phi[(size_t)a * nc + k], pb = phi[(size_t)b * nc + k];
    const double* ga = grad + ((size_t)a * nc + k) * 3;
    const double* gb = grad + ((size_t)b * nc + k) * 3;
    const double pa_aux = da(pa, dot3(ga[0], ga[1], ga[2], xa.x, xa.y, xa.z));
    const double pb_aux = da(pb, dot3(gb[0], gb[1], gb[2], xb.x, xb.y, xb.z));
    double r_cor = 0.0;
    if (c != 0.0) {
      double pf;
      if (scheme == 0) {
        pf = lerp(w, pb_aux, pa_aux);
      } else {
        const bool fwd = c > 0.0;
        const double pc = fwd ? pa_aux : pb_aux, pd = fwd ? pb_aux : pa_aux;
        const double* gc = fwd ? ga : gb;
        const double* xcA = g.xc + 3 * a;
        const double* xcB = g.xc + 3 * b;
        const double xpa[3] = {da(xcA[0], xa.x), da(xcA[1], xa.y), da(xcA[2], xa.z)};
        const double xpb[3] = {da(xcB[0], xb.x), da(xcB[1], xb.y), da(xcB[2], xb.z)};
        double dx[3];
        for (int q = 0; q < 3; ++q) dx[q] = fwd ? ds(xpb[q], xpa[q]) : ds(xpa[q], xpb[q]);
        const double pu = ds(pd, dm(2.0, dot3(gc[0], gc[1], gc[2], dx[0], dx[1], dx[2])));
        double r = dd(ds(pc, pu), da(ds(pd, pc), 1e-20));
        if (scheme == 1) {
          r = smax(0.0, smin(1.0, r));
        } else if (scheme == 2) {
          r = dd(da(r, fabs(r)), da(da(1.0, fabs(r)), 1e-20));
        } else {  // std::max({0, min(1, 2r), min(2, r)}): the first largest
          double m = 0.0;
          const double c1 = smin(1.0, dm(2.0, r)), c2 = smin(2.0, r);
          if (m < c1) m = c1;
          if (m < c2) m = c2;
          r = m;
        }
        pf = da(pc, dm(dm(0.5, r), ds(pd, pc)));
      }
      const double up = c > 0.0 ? pa : pb;
      r_cor = dm(dm(c_bl, c), ds(up, pf));
    }
    cor[t] = da(r_cor, dm(d, ds(ds(pb_aux, pa_aux), ds(pb, pa))));
  }
}

__global__ void k_fv_deferred_cells(Geo g, int nc, const double* __restrict__ cor,
                                    double* __restrict__ rhs) {
  const long long tot = (long long)g.n_cell * nc;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t / nc), k = (int)(t % nc);
    double acc = rhs[t];
    for (int q = g.cf_ptr[c]; q < g.cf_ptr[c + 1]; ++q) {
      const int f = g.cf[q];
      if (g.in[f] < 0) continue;
      const double x = cor[(size_t)f * nc + k];
      acc = g.ip[f] == c ? da(acc, x) : ds(acc, x);
    }
    rhs[t] = acc;
  }
}

// ---- Rhie-Chow face fluxes ------------------------------------------------------------
__global__ void k_fv_face_flux(Geo g, const double* __restrict__ u, const double* __restrict__ pr,
                               const double* __restrict__ gp, const double* __restrict__ ap,
                               double rho, int aux, double* __restrict__ flux) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < g.n_face; f += gridDim.x * blockDim.x) {
    const int a = g.ip[f], b = g.in[f];
    if (b < 0) {
      flux[f] = 0.0;
      continue;
    }
    const double w = g.w[f];
    const double* nn = g.nrm + 3 * f;
    const double ufx = lerp(w, u[3 * b], u[3 * a]), ufy = lerp(w, u[3 * b + 1], u[3 * a + 1]),
                 ufz = lerp(w, u[3 * b + 2], u[3 * a + 2]);
    const double d = pc_coef(g, f, a, b, ap, rho);
    const double gx = lerp(w, gp[3 * b], gp[3 * a]), gy = lerp(w, gp[3 * b + 1], gp[3 * a + 1]),
                 gz = lerp(w, gp[3 * b + 2], gp[3 * a + 2]);
    const double dx = ds(g.xc[3 * b], g.xc[3 * a]), dy = ds(g.xc[3 * b + 1], g.xc[3 * a + 1]),
                 dz = ds(g.xc[3 * b + 2], g.xc[3 * a + 2]);
    double pa = pr[a], pb = pr[b];
    if (aux) {  // cfd_setup.f90:611-614
      const Dx xa = aux_dx(g, f, a), xb = aux_dx(g, f, b);
      pa = da(pa, dot3(gp[3 * a], gp[3 * a + 1], gp[3 * a + 2], xa.x, xa.y, xa.z));
      pb = da(pb, dot3(gp[3 * b], gp[3 * b + 1], gp[3 * b + 2], xb.x, xb.y, xb.z));
    }
    const double dp = ds(ds(pb, pa), da(da(dm(gx, dx), dm(gy, dy)), dm(gz, dz)));
    const double un = da(da(dm(ufx, nn[0]), dm(ufy, nn[1])), dm(ufz, nn[2]));
    flux[f] = ds(dm(dm(rho, g.s[f]), un), dm(d, dp));
  }
}

// ---- mass imbalance -------------------------------------------------------------------
__global__ void k_fv_imbalance(Geo g, const double* __restrict__ flux, int pc,
                               double* __restrict__ bvec, double* __restrict__ part) {
  __shared__ double sh[kBlock / 32];
  double acc = 0.0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < g.n_cell; c += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int q = g.cf_ptr[c]; q < g.cf_ptr[c + 1]; ++q) {
      const int f = g.cf[q];
      if (g.in[f] < 0) continue;
      s = g.ip[f] == c ? ds(s, flux[f]) : da(s, flux[f]);
    }
    if (c == pc) s = 0.0;
    bvec[c] = s;
    acc += fabs(s);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < kBlock / 32; ++k) t += sh[k];
    part[blockIdx.x] = t;
  }
}

__global__ void k_fv_sum(int n, const double* __restrict__ part, double* __restrict__ out) {
  __shared__ double sh[kBlock / 32];
  double acc = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) acc += part[k];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < kBlock / 32; ++k) t += sh[k];
    *out = t;
  }
}

// ---- SIMPLE corrections -------------------------------------------------------------------
__global__ void k_fv_correct_cells(Geo g, const double* __restrict__ pp,
                                   const double* __restrict__ gpp, const double* __restrict__ ap,
                                   double urf_p, double* __restrict__ u, double* __restrict__ p) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < g.n_cell; c += gridDim.x * blockDim.x) {
    p[c] = da(p[c], dm(urf_p, pp[c]));
    const double k = dd(g.vol[c], da(ap[c], 1e-20));
    for (int d = 0; d < 3; ++d) u[3 * c + d] = ds(u[3 * c + d], dm(k, gpp[3 * c + d]));
  }
}

__global__ void k_fv_correct_faces(Geo g, const double* __restrict__ pp,
                                   const double* __restrict__ ap, double rho,
                                   double* __restrict__ flux) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < g.n_face; f += gridDim.x * blockDim.x) {
    const int a = g.ip[f], b = g.in[f];
    if (b < 0) continue;
    flux[f] = ds(flux[f], dm(pc_coef(g, f, a, b, ap, rho), ds(pp[b], pp[a])));
  }
}

struct DBuf {
  void* p = nullptr;
  ~DBuf() { if (p) cudaFree(p); }
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

}  // namespace

struct fv_gpu {
  int dev = 0;
  cudaStream_t stream = nullptr;
  Geo g{};
  DBuf ip, in, s, nrm, xf, l, w, xc, vol, vr, cf_ptr, cf, dface, part, total, tmp;
  size_t tmp_bytes = 0;
};

namespace {

template <typename T>
cudaError_t up(DBuf& b, const T* h, size_t count) {
  cudaError_t e = cudaMalloc(&b.p, std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess || count == 0) return e;
  return cudaMemcpy(b.p, h, count * sizeof(T), cudaMemcpyHostToDevice);
}

// The context's scratch of at least `bytes` (grown in order on its stream).
double* scratch(fv_gpu* fv, size_t bytes) {
  if (fv->tmp_bytes >= bytes && fv->tmp.p) return fv->tmp.as<double>();
  if (cudaStreamSynchronize(fv->stream) != cudaSuccess) return nullptr;
  if (fv->tmp.p) cudaFree(fv->tmp.p);
  fv->tmp.p = nullptr;
  fv->tmp_bytes = 0;
  if (cudaMalloc(&fv->tmp.p, bytes) != cudaSuccess) return nullptr;
  fv->tmp_bytes = bytes;
  return fv->tmp.as<double>();
}

int enter(fv_gpu* fv) {
  if (!fv) return SOLV_GPU_BAD_INPUT;
  return cudaSetDevice(fv->dev) == cudaSuccess ? SOLV_GPU_OK : SOLV_GPU_DEVICE_ERROR;
}

int done() {
  return cudaGetLastError() == cudaSuccess ? SOLV_GPU_OK : SOLV_GPU_DEVICE_ERROR;
}

}  // namespace

extern "C" {

int fv_gpu_create(fv_gpu** out, int device, int n_cell, int n_face, const int* ip, const int* in,
                  const double* area, const double* nrm, const double* xf, const double* l_pn,
                  const double* w_fp, const double* xc, const double* vol) {
  if (!out) return SOLV_GPU_BAD_INPUT;
  *out = nullptr;
  if (n_cell <= 0 || n_face < 0 || !ip || !in || !area || !nrm || !xf || !l_pn || !w_fp || !xc ||
      !vol)
    return SOLV_GPU_BAD_INPUT;
  std::vector<int> a(n_face), b(n_face), cnt(n_cell + 1, 0);
  for (int f = 0; f < n_face; ++f) {
    a[f] = ip[f] - 1;
    b[f] = in[f] - 1;
    if (a[f] < 0 || a[f] >= n_cell || b[f] < -1 || b[f] >= n_cell || a[f] == b[f])
      return SOLV_GPU_BAD_INPUT;
    cnt[a[f] + 1]++;
    if (b[f] >= 0) cnt[b[f] + 1]++;
  }
  for (int c = 0; c < n_cell; ++c) cnt[c + 1] += cnt[c];
  std::vector<int> cf(cnt[n_cell]);
  std::vector<int> pos(cnt.begin(), cnt.end() - 1);
  for (int f = 0; f < n_face; ++f) {  // ascending faces: each list comes out sorted
    cf[pos[a[f]]++] = f;
    if (b[f] >= 0) cf[pos[b[f]]++] = f;
  }
  if (cudaSetDevice(device) != cudaSuccess) return SOLV_GPU_DEVICE_ERROR;
  fv_gpu* fv = new fv_gpu;
  fv->dev = device;
  const size_t F = n_face, N = n_cell;
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
  chk(up(fv->ip, a.data(), F));
  chk(up(fv->in, b.data(), F));
  chk(up(fv->s, area, F));
  chk(up(fv->nrm, nrm, 3 * F));
  chk(up(fv->xf, xf, 3 * F));
  chk(up(fv->l, l_pn, F));
  chk(up(fv->w, w_fp, F));
  chk(up(fv->xc, xc, 3 * N));
  chk(up(fv->vol, vol, N));
  chk(up(fv->cf_ptr, cnt.data(), N + 1));
  chk(up(fv->cf, cf.data(), cf.size()));
  chk(cudaMalloc(&fv->dface.p, std::max<size_t>(F, 1) * sizeof(double)));
  chk(cudaMalloc(&fv->part.p, kRedBlocks * sizeof(double)));
  chk(cudaMalloc(&fv->total.p, sizeof(double)));
  chk(cudaMalloc(&fv->vr.p, std::max<size_t>(N, 1) * sizeof(double)));
  if (e == cudaSuccess) {
    k_fv_recip<<<grid(n_cell), kBlock>>>(n_cell, fv->vol.as<double>(), fv->vr.as<double>());
    chk(cudaGetLastError());
    chk(cudaDeviceSynchronize());
  }
  if (e != cudaSuccess) {
    delete fv;
    return SOLV_GPU_DEVICE_ERROR;
  }
  Geo& g = fv->g;
  g.n_cell = n_cell;
  g.n_face = n_face;
  g.ip = fv->ip.as<int>();
  g.in = fv->in.as<int>();
  g.s = fv->s.as<double>();
  g.nrm = fv->nrm.as<double>();
  g.xf = fv->xf.as<double>();
  g.l = fv->l.as<double>();
  g.w = fv->w.as<double>();
  g.xc = fv->xc.as<double>();
  g.vol = fv->vol.as<double>();
  g.cf_ptr = fv->cf_ptr.as<int>();
  g.cf = fv->cf.as<int>();
  *out = fv;
  return SOLV_GPU_OK;
}

int fv_gpu_destroy(fv_gpu* fv) {
  if (!fv) return SOLV_GPU_BAD_INPUT;
  cudaSetDevice(fv->dev);
  cudaStreamSynchronize(fv->stream);
  delete fv;
  return SOLV_GPU_OK;
}

int fv_gpu_set_stream(fv_gpu* fv, void* stream) {
  if (!fv) return SOLV_GPU_BAD_INPUT;
  fv->stream = static_cast<cudaStream_t>(stream);
  return SOLV_GPU_OK;
}

int fv_gpu_momentum(fv_gpu* fv, const double* u, const double* flux, double rho, double mu,
                    double u_lid, double urf, double* p, double* n, double* pl, double* rhs,
                    double* flux_out) {
  int rc = enter(fv);
  if (rc) return rc;
  if (!u || !p || !n || !pl || !(urf > 0.0)) return SOLV_GPU_BAD_INPUT;
  const Geo& g = fv->g;
  k_fv_mom_faces<<<grid(g.n_face), kBlock, 0, fv->stream>>>(g, u, flux, rho, mu, p, n, flux_out);
  k_fv_mom_cells<<<grid(g.n_cell), kBlock, 0, fv->stream>>>(g, u, p, n, u_lid, urf, pl, rhs);
  return done();
}

int fv_gpu_pressure_correction(fv_gpu* fv, const double* ap, double rho, int pin, double* p,
                               double* n, double* pl) {
  int rc = enter(fv);
  if (rc) return rc;
  if (!ap || !p || !n || !pl || pin < 0 || pin > fv->g.n_cell) return SOLV_GPU_BAD_INPUT;
  const Geo& g = fv->g;
  k_fv_pc_faces<<<grid(g.n_face), kBlock, 0, fv->stream>>>(g, ap, rho, pin - 1,
                                                           fv->dface.as<double>(), p, n);
  k_fv_pc_cells<<<grid(g.n_cell), kBlock, 0, fv->stream>>>(g, fv->dface.as<double>(), pl);
  return done();
}

int fv_gpu_gradient(fv_gpu* fv, int ncomp, const double* phi, double* grad) {
  int rc = enter(fv);
  if (rc) return rc;
  if (ncomp < 1 || ncomp > 16 || !phi || !grad) return SOLV_GPU_BAD_INPUT;
  const Geo& g = fv->g;
  k_fv_gradient<<<grid((long long)g.n_cell * ncomp), kBlock, 0, fv->stream>>>(g, ncomp, phi,
                                                                              grad);
  return done();
}

int fv_gpu_face_flux(fv_gpu* fv, const double* u, const double* p, const double* gradp,
                     const double* ap, double rho, double* flux) {
  int rc = enter(fv);
  if (rc) return rc;
  if (!u || !p || !gradp || !ap || !flux) return SOLV_GPU_BAD_INPUT;
  const Geo& g = fv->g;
  k_fv_face_flux<<<grid(g.n_face), kBlock, 0, fv->stream>>>(g, u, p, gradp, ap, rho, 0, flux);
  return done();
}

int fv_gpu_face_flux_aux(fv_gpu* fv, const double* u, const double* p, const double* gradp,
                         const double* ap, double rho, double* flux) {
  int rc = enter(fv);
  if (rc) return rc;
  if (!u || !p || !gradp || !ap || !flux) return SOLV_GPU_BAD_INPUT;
  const Geo& g = fv->g;
  k_fv_face_flux<<<grid(g.n_face), kBlock, 0, fv->stream>>>(g, u, p, gradp, ap, rho, 1, flux);
  return done();
}

int fv_gpu_gradient_sweeps(fv_gpu* fv, int ncomp, const double* phi, const double* bval,
                           int n_iter, int neu, double* grad) {
  int rc = enter(fv);
  if (rc) return rc;
  if (ncomp < 1 || ncomp > 16 || !phi || !grad || n_iter < 1 || n_iter > 64 || neu < 0 ||
      neu > 2 || (neu == 0 && !bval))
    return SOLV_GPU_BAD_INPUT;
  const Geo& g = fv->g;
  const size_t G = (size_t)3 * ncomp * g.n_cell;
  double* t = scratch(fv, n_iter > 1 ? 2 * G * sizeof(double) : sizeof(double));
  if (!t) return SOLV_GPU_DEVICE_ERROR;
  const double* g0 = nullptr;
  for (int it = 1; it <= n_iter; ++it) {
    double* out = it == n_iter ? grad : t + ((it & 1) ? 0 : G);
    k_fv_grad_sweep<<<grid((long long)g.n_cell * ncomp), kBlock, 0, fv->stream>>>(
        g, ncomp, phi, bval, neu, fv->vr.as<double>(), g0, out);
    g0 = out;
  }
  return done();
}

int fv_gpu_momentum_deferred(fv_gpu* fv, int ncomp, const double* phi, const double* grad,
                             const double* flux, double mu, double c_bl, int scheme,
                             double* rhs) {
  int rc = enter(fv);
  if (rc) return rc;
  if (ncomp < 1 || ncomp > 16 || !phi || !grad || !flux || !rhs || scheme < 0 || scheme > 3)
    return SOLV_GPU_BAD_INPUT;
  const Geo& g = fv->g;
  double* cor = scratch(fv, std::max<size_t>((size_t)g.n_face * ncomp, 1) * sizeof(double));
  if (!cor) return SOLV_GPU_DEVICE_ERROR;
  k_fv_deferred_faces<<<grid((long long)g.n_face * ncomp), kBlock, 0, fv->stream>>>(
      g, ncomp, phi, grad, flux, mu, c_bl, scheme, cor);
  k_fv_deferred_cells<<<grid((long long)g.n_cell * ncomp), kBlock, 0, fv->stream>>>(g, ncomp, cor,
                                                                                    rhs);
  return done();
}

int fv_gpu_mass_imbalance(fv_gpu* fv, const double* flux, int pin, double* b, double* total) {
  int rc = enter(fv);
  if (rc) return rc;
  if (!flux || !b || pin < 0 || pin > fv->g.n_cell) return SOLV_GPU_BAD_INPUT;
  const Geo& g = fv->g;
  const int nb = std::min(grid(g.n_cell), kRedBlocks);
  k_fv_imbalance<<<nb, kBlock, 0, fv->stream>>>(g, flux, pin - 1, b, fv->part.as<double>());
  k_fv_sum<<<1, kBlock, 0, fv->stream>>>(nb, fv->part.as<double>(), fv->total.as<double>());
  if ((rc = done())) return rc;
  if (total) {
    if (cudaMemcpyAsync(total, fv->total.p, sizeof(double), cudaMemcpyDeviceToHost, fv->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(fv->stream) != cudaSuccess)
      return SOLV_GPU_DEVICE_ERROR;
  }
  return SOLV_GPU_OK;
}

int fv_gpu_simple_correct(fv_gpu* fv, const double* pp, const double* gradpp, const double* ap,
                          double rho, double urf_p, double* u, double* p, double* flux) {
  int rc = enter(fv);
  if (rc) return rc;
  if (!pp || !gradpp || !ap || !u || !p || !flux) return SOLV_GPU_BAD_INPUT;
  const Geo& g = fv->g;
  k_fv_correct_cells<<<grid(g.n_cell), kBlock, 0, fv->stream>>>(g, pp, gradpp, ap, urf_p, u, p);
  k_fv_correct_faces<<<grid(g.n_face), kBlock, 0, fv->stream>>>(g, pp, ap, rho, flux);
  return done();
}

}  // extern "C"
