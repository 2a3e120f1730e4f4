// fvmesh.cpp -- host-side hex mesh generation, Gambit reading, renumbering,
// face-list emission and matrix assembly for the face-addressed solvers.
//
// Connectivity: spray-simulation/grd_conn.f90:45-152.  Geometry:
// spray-simulation/grd_geom.f90:31-43, 119-208.  Coefficients:
// spray-simulation/cfd_setup.f90:324-330 (momentum, upwind) and
// cfd_setup.f90:604-646 (pressure correction; here with unit density,
// unit d-coefficient so the face coefficient is area / l_pn).
#include "fvmesh.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <numeric>
#include <random>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

namespace {

// Brick element, Gambit vertex order (x fastest): local faces as vertex
// lists, outward normals by the right-hand rule.  This is the Gambit
// "brick" face table the reference reads from gambit.vrt (type 4); it is a
// file-format fact, so it is the same here.
constexpr int kHexFaces[6][4] = {{0, 1, 5, 4}, {1, 3, 7, 5}, {3, 2, 6, 7},
                                 {2, 0, 4, 6}, {1, 0, 2, 3}, {4, 5, 7, 6}};

struct V3 {
  double x, y, z;
};
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline double mag(V3 a) { return std::sqrt(dot(a, a)); }

}  // namespace

struct fvm_mesh {
  std::vector<V3> vert;
  std::vector<int32_t> cell_vert;  // 8 per cell, 0-based vertex ids
  std::vector<int32_t> cell_nbr;   // 6 per cell, 0-based cell id or -1
  // derived face list (0-based owner/neighbour, local face of the owner)
  std::vector<int32_t> f_ip, f_in;
  std::vector<int8_t> f_loc;
  std::vector<V3> xc;              // cell centres
  int n_cell = 0;
  int n_bface = 0;
  // face distance and interpolation weight: false = along the face normal
  // between the auxiliary points (the linear weight), true = the
  // reference's centre distance and 1 - |x_f - x_P| / l_pn
  bool ref_weights = false;
  // optional cache of the face geometry (9 doubles per face) and volumes,
  // for repeated assembly on one mesh (fvm_mesh_cache_geometry)
  std::vector<double> geo, vol_cache;

  void emit_faces() {
    geo.clear();
    vol_cache.clear();
    f_ip.clear();
    f_in.clear();
    f_loc.clear();
    n_bface = 0;
    size_t est = (size_t)n_cell * 3 + 64;
    f_ip.reserve(est);
    f_in.reserve(est);
    f_loc.reserve(est);
    for (int c = 0; c < n_cell; ++c) {
      for (int k = 0; k < 6; ++k) {
        int nb = cell_nbr[(size_t)c * 6 + k];
        if (nb >= 0 && nb < c) continue;  // already emitted by the lower cell
        f_ip.push_back(c);
        f_in.push_back(nb);  // -1 = boundary
        f_loc.push_back((int8_t)k);
        if (nb < 0) ++n_bface;
      }
    }
  }

  void centres() {
    xc.resize(n_cell);
    for (int c = 0; c < n_cell; ++c) {
      V3 s{0, 0, 0};
      for (int v = 0; v < 8; ++v) s = s + vert[cell_vert[(size_t)c * 8 + v]];
      xc[c] = s * (1.0 / 8.0);
    }
  }

  // grd_geom.f90:119-147 (3-d branch) and :161-198.
  void face_geom(size_t f, double &s, V3 &nrm, V3 &xf, double &l_pn,
                 double &w_fp) const {
    if (!geo.empty()) {
      const double *g = &geo[9 * f];
      s = g[0];
      nrm = {g[1], g[2], g[3]};
      xf = {g[4], g[5], g[6]};
      l_pn = g[7];
      w_fp = g[8];
      return;
    }
    int c = f_ip[f];
    int k = f_loc[f];
    V3 v[4];
    for (int i = 0; i < 4; ++i) v[i] = vert[cell_vert[(size_t)c * 8 + kHexFaces[k][i]]];
    // Area vector of the quadrilateral: 1/2 sum v_i x v_{i+1}.  It does not
    // depend on where a triangulation starts, so a face is the same seen
    // from either cell and every cell's area vectors sum to zero.  The
    // reference's fan triangles with averaged unit normals
    // (grd_geom.f90:127-140) do not close on non-planar (jittered) faces,
    // which puts a spurious O(jitter/h) gradient on a constant field.
    V3 A{0, 0, 0};
    for (int i = 0; i < 4; ++i) A = A + cross(v[i], v[(i + 1) & 3]);
    A = A * 0.5;
    s = mag(A);
    nrm = A * (1.0 / s);
    xf = (v[0] + v[1] + v[2] + v[3]) * 0.25;
    V3 xp_aux = xf - nrm * dot(xf - xc[c], nrm);
    int nb = f_in[f];
    if (ref_weights) {  // cfd_grid.f90:520, 524, 534
      l_pn = nb >= 0 ? mag(xc[nb] - xc[c]) : mag(xf - xc[c]);
      w_fp = nb >= 0 ? 1.0 - mag(xf - xc[c]) / l_pn : 1.0;
    } else if (nb >= 0) {
      V3 xn_aux = xf - nrm * dot(xf - xc[nb], nrm);
      l_pn = mag(xn_aux - xp_aux);
      w_fp = mag(xf - xp_aux) / l_pn;
    } else {
      l_pn = mag(xf - xp_aux);
      w_fp = 1.0;
    }
  }
};

extern "C" {

fvm_mesh *fvm_mesh_hex(int nx, int ny, int nz, double jitter, uint64_t seed,
                       int permute) {
  if (nx < 1 || ny < 1 || nz < 1) return nullptr;
  auto *m = new fvm_mesh();
  std::mt19937_64 rng(seed);
  auto uni = [&rng]() {  // [-1, 1)
    return (double)(rng() >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
  };
  const int vx = nx + 1, vy = ny + 1, vz = nz + 1;
  const double hx = 1.0 / nx, hy = 1.0 / ny, hz = 1.0 / nz;
  m->vert.resize((size_t)vx * vy * vz);
  for (int k = 0; k < vz; ++k)
    for (int j = 0; j < vy; ++j)
      for (int i = 0; i < vx; ++i) {
        V3 x{i * hx, j * hy, k * hz};
        bool interior = i > 0 && i < nx && j > 0 && j < ny && k > 0 && k < nz;
        double dx = uni(), dy = uni(), dz = uni();
        if (interior) {
          x.x += jitter * hx * dx;
          x.y += jitter * hy * dy;
          x.z += jitter * hz * dz;
        }
        m->vert[((size_t)k * vy + j) * vx + i] = x;
      }
  const int N = nx * ny * nz;
  m->n_cell = N;
  // lexicographic cell id -> stored cell id
  std::vector<int32_t> id(N);
  std::iota(id.begin(), id.end(), 0);
  if (permute) {
    for (int i = N - 1; i > 0; --i) {
      uint64_t r = rng() % (uint64_t)(i + 1);
      std::swap(id[i], id[(int)r]);
    }
  }
  m->cell_vert.resize((size_t)N * 8);
  m->cell_nbr.assign((size_t)N * 6, -1);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        int lex = (k * ny + j) * nx + i;
        int c = id[lex];
        int32_t *cv = &m->cell_vert[(size_t)c * 8];
        for (int b = 0; b < 8; ++b) {
          int di = b & 1, dj = (b >> 1) & 1, dk = (b >> 2) & 1;
          cv[b] = ((k + dk) * vy + (j + dj)) * vx + (i + di);
        }
        int32_t *cn = &m->cell_nbr[(size_t)c * 6];
        // local face order: -y, +x, +y, -x, -z, +z
        cn[0] = j > 0 ? id[lex - nx] : -1;
        cn[1] = i < nx - 1 ? id[lex + 1] : -1;
        cn[2] = j < ny - 1 ? id[lex + nx] : -1;
        cn[3] = i > 0 ? id[lex - 1] : -1;
        cn[4] = k > 0 ? id[lex - nx * ny] : -1;
        cn[5] = k < nz - 1 ? id[lex + nx * ny] : -1;
      }
  m->centres();
  m->emit_faces();
  return m;
}

fvm_mesh *fvm_mesh_read_neu(const char *path) {
  std::ifstream in(path);
  if (!in) return nullptr;
  auto *m = new fvm_mesh();
  std::string line;
  int n_vrt = 0, n_vol = 0, dim = 3;
  bool ok_sizes = false;
  while (std::getline(in, line)) {
    if (line.find("NUMNP") != std::string::npos) {
      std::getline(in, line);
      std::istringstream ss(line);
      int n_grp = 0, n_bset = 0, ndfcd = 3;
      ss >> n_vrt >> n_vol >> n_grp >> n_bset >> ndfcd;
      dim = ndfcd == 2 ? 2 : 3;
      ok_sizes = n_vrt > 0 && n_vol > 0;
    } else if (line.find("NODAL COORDINATES") != std::string::npos && ok_sizes) {
      // a 2-d mesh gets a second copy of its nodes one unit deep
      m->vert.resize((size_t)n_vrt * (dim == 2 ? 2 : 1));
      for (int i = 0; i < n_vrt; ++i) {
        int idx;
        double x, y, z = 0.0;
        in >> idx >> x >> y;
        if (dim == 3) in >> z;
        if (!in || idx < 1 || idx > n_vrt) { delete m; return nullptr; }
        m->vert[idx - 1] = {x, y, z};
        if (dim == 2) m->vert[(size_t)n_vrt + idx - 1] = {x, y, 1.0};
      }
    } else if (line.find("ELEMENTS/CELLS") != std::string::npos && ok_sizes) {
      m->n_cell = n_vol;
      m->cell_vert.resize((size_t)n_vol * 8);
      std::vector<char> seen(n_vol, 0);
      const int want_ty = dim == 2 ? 2 : 4, want_nv = dim == 2 ? 4 : 8;
      for (int e = 0; e < n_vol; ++e) {
        int idx, ty, nv;
        in >> idx >> ty >> nv;
        if (!in || ty != want_ty || nv != want_nv || idx < 1 || idx > n_vol || seen[idx - 1]) {
          delete m;  // bricks (3-d) or quadrilaterals (2-d), each numbered once
          return nullptr;
        }
        seen[idx - 1] = 1;
        int g[8];
        for (int v = 0; v < nv; ++v) {
          in >> g[v];
          if (!in || g[v] < 1 || g[v] > n_vrt) { delete m; return nullptr; }
          g[v] -= 1;
        }
        int32_t *cv = &m->cell_vert[(size_t)(idx - 1) * 8];
        if (dim == 3) {
          for (int v = 0; v < 8; ++v) cv[v] = g[v];
        } else {
          // the quadrilateral n1..n4 (in order around it) as the brick one
          // unit deep in the brick's vertex order (x fastest): counter-
          // clockwise seen from +z so that the brick's volume is positive
          if (m->vert.size() < (size_t)2 * n_vrt) { delete m; return nullptr; }
          double a2 = 0.0;
          for (int v = 0; v < 4; ++v) {
            const V3 p = m->vert[g[v]], q = m->vert[g[(v + 1) & 3]];
            a2 += p.x * q.y - q.x * p.y;
          }
          if (a2 < 0.0) std::swap(g[1], g[3]);
          const int lo[4] = {g[0], g[1], g[3], g[2]};
          for (int v = 0; v < 4; ++v) {
            cv[v] = lo[v];
            cv[v + 4] = lo[v] + n_vrt;
          }
        }
      }
    }
  }
  if (m->n_cell == 0 || m->vert.empty()) { delete m; return nullptr; }
  for (int32_t g : m->cell_vert)
    if (g < 0 || (size_t)g >= m->vert.size()) { delete m; return nullptr; }
  // hashed face matching: key = sorted vertex quadruple
  m->cell_nbr.assign((size_t)m->n_cell * 6, -1);
  struct Key {
    std::array<int32_t, 4> v;
    bool operator==(const Key &o) const { return v == o.v; }
  };
  struct H {
    size_t operator()(const Key &k) const {
      uint64_t h = 1469598103934665603ull;
      for (int x : k.v) { h ^= (uint64_t)(uint32_t)x; h *= 1099511628211ull; }
      return (size_t)h;
    }
  };
  std::unordered_map<Key, int64_t, H> open;
  open.reserve((size_t)m->n_cell * 4);
  for (int c = 0; c < m->n_cell; ++c)
    for (int k = 0; k < 6; ++k) {
      Key key;
      for (int i = 0; i < 4; ++i) key.v[i] = m->cell_vert[(size_t)c * 8 + kHexFaces[k][i]];
      std::sort(key.v.begin(), key.v.end());
      auto it = open.find(key);
      if (it == open.end()) {
        open.emplace(key, (int64_t)c * 6 + k);
      } else {
        int64_t o = it->second;
        m->cell_nbr[(size_t)o] = c;
        m->cell_nbr[(size_t)c * 6 + k] = (int)(o / 6);
        open.erase(it);
      }
    }
  m->centres();
  m->emit_faces();
  return m;
}

void fvm_mesh_free(fvm_mesh *m) { delete m; }

void fvm_mesh_sizes(const fvm_mesh *m, int *n_cell, int *n_face, int *n_bface,
                    int *n_vert) {
  if (n_cell) *n_cell = m->n_cell;
  if (n_face) *n_face = (int)m->f_ip.size();
  if (n_bface) *n_bface = m->n_bface;
  if (n_vert) *n_vert = (int)m->vert.size();
}

void fvm_mesh_faces(const fvm_mesh *m, int *ip, int *in) {
  size_t F = m->f_ip.size();
  for (size_t f = 0; f < F; ++f) {
    ip[f] = m->f_ip[f] + 1;
    in[f] = m->f_in[f] + 1;  // -1 -> 0
  }
}

void fvm_mesh_face_geom(const fvm_mesh *m, double *s, double *nrm, double *xf,
                        double *l_pn, double *w_fp) {
  size_t F = m->f_ip.size();
  for (size_t f = 0; f < F; ++f) {
    double a, l, w;
    V3 nn, x;
    m->face_geom(f, a, nn, x, l, w);
    if (s) s[f] = a;
    if (nrm) { nrm[3 * f] = nn.x; nrm[3 * f + 1] = nn.y; nrm[3 * f + 2] = nn.z; }
    if (xf) { xf[3 * f] = x.x; xf[3 * f + 1] = x.y; xf[3 * f + 2] = x.z; }
    if (l_pn) l_pn[f] = l;
    if (w_fp) w_fp[f] = w;
  }
}

void fvm_mesh_set_face_weights(fvm_mesh *m, int reference) {
  const bool cached = !m->geo.empty();
  m->ref_weights = reference != 0;
  m->geo.clear();
  if (cached) fvm_mesh_cache_geometry(m);
}

void fvm_mesh_cache_geometry(fvm_mesh *m) {
  const size_t F = m->f_ip.size();
  std::vector<double> g(9 * F);
  for (size_t f = 0; f < F; ++f) {
    double s, l, w;
    V3 nn, x;
    m->face_geom(f, s, nn, x, l, w);
    double *q = &g[9 * f];
    q[0] = s; q[1] = nn.x; q[2] = nn.y; q[3] = nn.z; q[4] = x.x; q[5] = x.y; q[6] = x.z;
    q[7] = l; q[8] = w;
  }
  std::vector<double> v(m->n_cell);
  fvm_mesh_cell_geom(m, nullptr, v.data());
  m->geo.swap(g);
  m->vol_cache.swap(v);
}

void fvm_mesh_cell_geom(const fvm_mesh *m, double *xc, double *vol) {
  for (int c = 0; c < m->n_cell; ++c)
    if (xc) { xc[3 * c] = m->xc[c].x; xc[3 * c + 1] = m->xc[c].y; xc[3 * c + 2] = m->xc[c].z; }
  if (vol && !m->vol_cache.empty()) {
    std::copy(m->vol_cache.begin(), m->vol_cache.end(), vol);
    return;
  }
  if (vol) {
    // Volume of the cell whose faces are split into four triangles about
    // the face centre: tetrahedra from the cell centre to each triangle of
    // its own (outward) local faces.  The split does not depend on which
    // side describes the face, so the volumes add up to the domain exactly.
    // The reference's sum of x_f * s * n_x over faces (grd_geom.f90:150,
    // 172) uses averaged fan normals and global coordinates; its error
    // scales like h^2 while the volume scales like h^3, so on fine jittered
    // meshes (48^3 and up) it turns cell volumes negative.
    for (int c = 0; c < m->n_cell; ++c) {
      const V3 xc = m->xc[c];
      double v6 = 0.0;
      for (int k = 0; k < 6; ++k) {
        V3 q[4];
        for (int i = 0; i < 4; ++i) q[i] = m->vert[m->cell_vert[(size_t)c * 8 + kHexFaces[k][i]]];
        const V3 fc = (q[0] + q[1] + q[2] + q[3]) * 0.25;
        for (int t = 0; t < 4; ++t)
          v6 += dot(cross(q[t] - fc, q[(t + 1) & 3] - fc), fc - xc);
      }
      vol[c] = v6 / 6.0;
    }
  }
}

int fvm_mesh_renumber(fvm_mesh *m, int method, int *perm) {
  const int N = m->n_cell;
  std::vector<int32_t> order;  // order[new] = old
  order.reserve(N);
  if (method == 4) {
    // Multicolour: reverse Cuthill-McKee first (locality), then a greedy
    // colouring in that order (smallest colour no coloured neighbour has),
    // then cells colour by colour, each colour in RCM order.  The lower
    // triangle then couples only earlier colours, so the DIC / DILU
    // recurrences are as deep as the number of colours (2 for a hex mesh:
    // its face graph is bipartite and RCM visits it level by level).
    std::vector<int> rcm(N);
    if (fvm_mesh_renumber(m, 1, rcm.data()) != 0) return -1;
    std::vector<int> colour(N, -1);
    int nc = 0;
    for (int c = 0; c < N; ++c) {
      unsigned used = 0;
      for (int k = 0; k < 6; ++k) {
        const int nb = m->cell_nbr[(size_t)c * 6 + k];
        if (nb >= 0 && colour[nb] >= 0 && colour[nb] < 32) used |= 1u << colour[nb];
      }
      int col = 0;
      while (col < 32 && (used >> col & 1u)) ++col;
      colour[c] = col;
      nc = std::max(nc, col + 1);
    }
    order.resize(N);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return colour[a] < colour[b]; });
    std::vector<int32_t> second(N);
    for (int i = 0; i < N; ++i) second[order[i]] = i + 1;
    if (fvm_mesh_renumber(m, 3, second.data()) != 0) return -1;
    if (perm)
      for (int c = 0; c < N; ++c) perm[c] = second[rcm[c] - 1];
    return 0;
  }
  if (method == 1) {
    // Reverse Cuthill-McKee: BFS from a pseudo-peripheral cell (repeated
    // BFS to the farthest, least-connected cell), neighbours by degree.
    auto degree = [&](int c) {
      int d = 0;
      for (int k = 0; k < 6; ++k) d += m->cell_nbr[(size_t)c * 6 + k] >= 0;
      return d;
    };
    std::vector<int32_t> level(N, -1);
    auto bfs_far = [&](int start) {
      std::fill(level.begin(), level.end(), -1);
      std::vector<int32_t> q;
      q.reserve(N);
      q.push_back(start);
      level[start] = 0;
      for (size_t h = 0; h < q.size(); ++h) {
        int c = q[h];
        for (int k = 0; k < 6; ++k) {
          int nb = m->cell_nbr[(size_t)c * 6 + k];
          if (nb >= 0 && level[nb] < 0) { level[nb] = level[c] + 1; q.push_back(nb); }
        }
      }
      int best = q.back(), bl = level[best], bd = degree(best);
      for (int c : q)
        if (level[c] == bl && degree(c) < bd) { best = c; bd = degree(c); }
      return std::make_pair(best, bl);
    };
    std::vector<char> seen(N, 0);
    for (int s0 = 0; s0 < N; ++s0) {
      if (seen[s0]) continue;
      int root = s0;
      auto r = bfs_far(root);
      for (int it = 0; it < 4; ++it) {
        auto r2 = bfs_far(r.first);
        if (r2.second <= r.second) break;
        r = r2;
      }
      root = r.first;
      size_t h = order.size();
      order.push_back(root);
      seen[root] = 1;
      for (; h < order.size(); ++h) {
        int c = order[h];
        int nb[6], nn = 0;
        for (int k = 0; k < 6; ++k) {
          int x = m->cell_nbr[(size_t)c * 6 + k];
          if (x >= 0 && !seen[x]) nb[nn++] = x;
        }
        std::stable_sort(nb, nb + nn, [&](int a, int b) { return degree(a) < degree(b); });
        for (int i = 0; i < nn; ++i) { seen[nb[i]] = 1; order.push_back(nb[i]); }
      }
    }
    std::reverse(order.begin(), order.end());
  } else if (method == 2) {
    // Morton (Z-order) key of the cell centre, 21 bits per axis.
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (const V3 &x : m->xc) {
      lo[0] = std::min(lo[0], x.x); hi[0] = std::max(hi[0], x.x);
      lo[1] = std::min(lo[1], x.y); hi[1] = std::max(hi[1], x.y);
      lo[2] = std::min(lo[2], x.z); hi[2] = std::max(hi[2], x.z);
    }
    auto spread = [](uint64_t v) {
      v &= 0x1fffff;
      v = (v | v << 32) & 0x1f00000000ffffull;
      v = (v | v << 16) & 0x1f0000ff0000ffull;
      v = (v | v << 8) & 0x100f00f00f00f00full;
      v = (v | v << 4) & 0x10c30c30c30c30c3ull;
      v = (v | v << 2) & 0x1249249249249249ull;
      return v;
    };
    std::vector<uint64_t> key(N);
    for (int c = 0; c < N; ++c) {
      uint64_t q[3];
      const double xs[3] = {m->xc[c].x, m->xc[c].y, m->xc[c].z};
      for (int d = 0; d < 3; ++d) {
        double t = (xs[d] - lo[d]) / std::max(hi[d] - lo[d], 1e-300);
        q[d] = (uint64_t)std::min(2097151.0, std::max(0.0, t * 2097151.0));
      }
      key[c] = spread(q[0]) | spread(q[1]) << 1 | spread(q[2]) << 2;
    }
    order.resize(N);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return key[a] < key[b]; });
  } else if (method == 3) {
    if (!perm) return -1;
    order.assign(N, -1);
    for (int c = 0; c < N; ++c) {
      int nw = perm[c] - 1;
      if (nw < 0 || nw >= N || order[nw] >= 0) return -1;
      order[nw] = c;
    }
  } else {
    return -1;
  }
  std::vector<int32_t> newid(N);
  for (int i = 0; i < N; ++i) newid[order[i]] = i;
  std::vector<int32_t> cv((size_t)N * 8), cn((size_t)N * 6);
  std::vector<V3> xc(N);
  for (int i = 0; i < N; ++i) {
    int o = order[i];
    std::memcpy(&cv[(size_t)i * 8], &m->cell_vert[(size_t)o * 8], 8 * sizeof(int32_t));
    for (int k = 0; k < 6; ++k) {
      int nb = m->cell_nbr[(size_t)o * 6 + k];
      cn[(size_t)i * 6 + k] = nb >= 0 ? newid[nb] : -1;
    }
    xc[i] = m->xc[o];
  }
  m->cell_vert.swap(cv);
  m->cell_nbr.swap(cn);
  m->xc.swap(xc);
  m->emit_faces();
  if (perm && method != 3)
    for (int c = 0; c < N; ++c) perm[c] = newid[c] + 1;
  return 0;
}

void fvm_assemble_pressure(const fvm_mesh *m, int pin, double *p, double *n,
                           double *pl) {
  const int N = m->n_cell;
  const size_t F = m->f_ip.size();
  for (int c = 0; c < N; ++c) pl[c] = 0.0;
  const int pc = pin - 1;
  for (size_t f = 0; f < F; ++f) {
    p[f] = 0.0;
    n[f] = 0.0;
    int a = m->f_ip[f], b = m->f_in[f];
    if (b < 0) continue;  // all-Neumann boundary
    double s, l, w;
    V3 nn, x;
    m->face_geom(f, s, nn, x, l, w);
    double d = s / l;
    pl[a] += d;
    pl[b] += d;
    if (a == pc || b == pc) continue;  // pinned cell: drop both couplings
    p[f] = -d;
    n[f] = -d;
  }
}

double fvm_assemble_momentum(const fvm_mesh *m, double gamma, double pe_max,
                             double cfl, double *p, double *n, double *pl) {
  const int N = m->n_cell;
  const size_t F = m->f_ip.size();
  // cell size from the mean volume
  double h = std::cbrt(1.0 / (double)N);
  const double U0 = pe_max * gamma / h;
  const double dt = cfl * h / U0;
  const double tp = 2.0 * M_PI;
  std::vector<double> vol(N);
  fvm_mesh_cell_geom(m, nullptr, vol.data());
  for (int c = 0; c < N; ++c) pl[c] = 0.0;
  for (size_t f = 0; f < F; ++f) {
    double s, l, w;
    V3 nn, x;
    m->face_geom(f, s, nn, x, l, w);
    int a = m->f_ip[f], b = m->f_in[f];
    double d = gamma * s / l;
    double u = U0 * std::sin(tp * x.x) * std::cos(tp * x.y) * std::cos(tp * x.z);
    double v = -U0 * std::cos(tp * x.x) * std::sin(tp * x.y) * std::cos(tp * x.z);
    double c = s * (u * nn.x + v * nn.y);
    if (b >= 0) {
      p[f] = -d + std::min(c, 0.0);
      n[f] = -d - std::max(c, 0.0);
      pl[a] -= p[f];
      pl[b] -= n[f];
    } else {
      p[f] = -d;  // wall: zero flux, Dirichlet diffusion
      n[f] = 0.0;
      pl[a] -= p[f];
    }
  }
  for (int c = 0; c < N; ++c) pl[c] += vol[c] / dt;
  return dt;
}

void fvm_cavity_field(const fvm_mesh *m, double u_lid, double *u) {
  // psi = a x^2 (1-x)^2 y^2 (1-y); dpsi/dy at (0.5, 1) = a * 1/16 * (2y - 3y^2)|_1 = -a/16
  const double a = -16.0 * u_lid;
  for (int c = 0; c < m->n_cell; ++c) {
    const double x = m->xc[c].x, y = m->xc[c].y, z = m->xc[c].z;
    const double fx = x * x * (1 - x) * (1 - x), dfx = 2 * x * (1 - x) * (1 - 2 * x);
    const double gy = y * y * (1 - y), dgy = 2 * y - 3 * y * y;
    const double hz = std::sin(M_PI * z);
    u[3 * c] = a * fx * dgy * hz;
    u[3 * c + 1] = -a * dfx * gy * hz;
    u[3 * c + 2] = 0.0;
  }
}

void fvm_assemble_momentum_field(const fvm_mesh *m, const double *u, const double *flux,
                                 double rho, double mu, double u_lid, double urf, double *p,
                                 double *n, double *pl, double *rhs, double *flux_out) {
  const int N = m->n_cell;
  const size_t F = m->f_ip.size();
  for (int c = 0; c < N; ++c) pl[c] = 0.0;
  if (rhs)
    for (size_t k = 0; k < 3 * (size_t)N; ++k) rhs[k] = 0.0;
  for (size_t f = 0; f < F; ++f) {
    double s, l, w;
    V3 nn, x;
    m->face_geom(f, s, nn, x, l, w);
    const int a = m->f_ip[f], b = m->f_in[f];
    const double d = mu * s / l;
    if (b >= 0) {
      double c;
      if (flux) {
        c = flux[f];
      } else {  // linear interpolation of u to the face (cfd_setup.f90:197-203)
        const double uf = w * u[3 * b] + (1 - w) * u[3 * a];
        const double vf = w * u[3 * b + 1] + (1 - w) * u[3 * a + 1];
        const double wf = w * u[3 * b + 2] + (1 - w) * u[3 * a + 2];
        c = rho * s * (uf * nn.x + vf * nn.y + wf * nn.z);
      }
      if (flux_out) flux_out[f] = c;
      p[f] = -d + std::min(c, 0.0);
      n[f] = -d - std::max(c, 0.0);
      pl[a] -= p[f];
      pl[b] -= n[f];
    } else {
      if (flux_out) flux_out[f] = 0.0;
      p[f] = -d;  // no-slip wall: Dirichlet diffusion, zero flux
      n[f] = 0.0;
      pl[a] += d;
      // the moving lid: the y = 1 wall (outward normal +y)
      if (rhs && nn.y > 0.9 && x.y > 1.0 - 1e-9) rhs[3 * a] += d * u_lid;
    }
  }
  // under-relaxation (cfd_setup.f90:517-518)
  for (int c = 0; c < N; ++c) {
    pl[c] = pl[c] / urf;
    if (rhs)
      for (int k = 0; k < 3; ++k) rhs[3 * c + k] += (1.0 - urf) * pl[c] * u[3 * c + k];
  }
}

void fvm_assemble_pressure_correction(const fvm_mesh *m, const double *ap, double rho, int pin,
                                      double *p, double *n, double *pl) {
  const int N = m->n_cell;
  const size_t F = m->f_ip.size();
  std::vector<double> vol(N);
  fvm_mesh_cell_geom(m, nullptr, vol.data());
  for (int c = 0; c < N; ++c) pl[c] = 0.0;
  const int pc = pin - 1;
  for (size_t f = 0; f < F; ++f) {
    p[f] = 0.0;
    n[f] = 0.0;
    const int a = m->f_ip[f], b = m->f_in[f];
    if (b < 0) continue;
    double s, l, w;
    V3 nn, x;
    m->face_geom(f, s, nn, x, l, w);
    const double p_r = w / (ap[b] + 1e-20) + (1 - w) / (ap[a] + 1e-20);
    const double v = w * vol[b] + (1 - w) * vol[a];
    const double d = rho * p_r * s * v / l;
    pl[a] += d;
    pl[b] += d;
    if (a == pc || b == pc) continue;
    p[f] = -d;
    n[f] = -d;
  }
}

void fvm_gradient(const fvm_mesh *m, int ncomp, const double *phi, double *grad) {
  const int N = m->n_cell;
  const size_t F = m->f_ip.size();
  std::vector<double> vol(N);
  fvm_mesh_cell_geom(m, nullptr, vol.data());
  std::fill(grad, grad + (size_t)3 * ncomp * N, 0.0);
  for (size_t f = 0; f < F; ++f) {
    double s, l, w;
    V3 nn, x;
    m->face_geom(f, s, nn, x, l, w);
    const int a = m->f_ip[f], b = m->f_in[f];
    for (int k = 0; k < ncomp; ++k) {
      const double pa = phi[(size_t)a * ncomp + k];
      const double pf = b >= 0 ? w * phi[(size_t)b * ncomp + k] + (1 - w) * pa : pa;
      double *ga = grad + ((size_t)a * ncomp + k) * 3;
      ga[0] += pf * s * nn.x;
      ga[1] += pf * s * nn.y;
      ga[2] += pf * s * nn.z;
      if (b >= 0) {
        double *gb = grad + ((size_t)b * ncomp + k) * 3;
        gb[0] -= pf * s * nn.x;
        gb[1] -= pf * s * nn.y;
        gb[2] -= pf * s * nn.z;
      }
    }
  }
  for (int c = 0; c < N; ++c)
    for (int k = 0; k < 3 * ncomp; ++k) grad[(size_t)c * 3 * ncomp + k] /= vol[c];
}

int fvm_gradient_sweeps(const fvm_mesh *m, int ncomp, const double *phi, const double *bval,
                        int n_iter, int neu, double *grad) {
  if (n_iter < 1 || neu < 0 || neu > 2 || (neu == 0 && !bval) || ncomp < 1) return -1;
  const int N = m->n_cell;
  const size_t F = m->f_ip.size(), G = (size_t)3 * ncomp * N;
  std::vector<double> vol(N), v_r(N);
  fvm_mesh_cell_geom(m, nullptr, vol.data());
  for (int c = 0; c < N; ++c) v_r[c] = 1.0 / vol[c];  // cfd_grid.f90:546
  // displacement of a cell centre to its auxiliary point on the face normal
  auto aux = [](V3 xf, V3 nn, V3 xc) { return (xf - nn * dot(xf - xc, nn)) - xc; };
  std::vector<double> g0(n_iter > 1 ? G : 0);
  for (int iter = 1; iter <= n_iter; ++iter) {
    std::fill(grad, grad + G, 0.0);
    for (size_t f = 0; f < F; ++f) {
      double s, l, w;
      V3 nn, xf;
      m->face_geom(f, s, nn, xf, l, w);
      const int a = m->f_ip[f], b = m->f_in[f];
      const V3 xa = m->xc[a];
      for (int k = 0; k < ncomp; ++k) {
        const double pa = phi[(size_t)a * ncomp + k];
        const double *ga0 = iter > 1 ? &g0[((size_t)a * ncomp + k) * 3] : nullptr;
        double pf;
        if (b >= 0) {
          const double pb = phi[(size_t)b * ncomp + k];
          if (iter > 1) {
            const double *gb0 = &g0[((size_t)b * ncomp + k) * 3];
            const double pp = pa + dot({ga0[0], ga0[1], ga0[2]}, aux(xf, nn, xa));
            const double pn = pb + dot({gb0[0], gb0[1], gb0[2]}, aux(xf, nn, m->xc[b]));
            pf = w * pn + (1.0 - w) * pp;
          } else {
            pf = w * pb + (1.0 - w) * pa;
          }
        } else if (neu > 0) {
          pf = pa;
          if (iter > 1 && neu == 2) pf = pf + dot({ga0[0], ga0[1], ga0[2]}, xf - xa);
        } else {
          pf = bval[f * ncomp + k];
        }
        const double ps = pf * s;
        double *ga = grad + ((size_t)a * ncomp + k) * 3;
        ga[0] += ps * nn.x * v_r[a];
        ga[1] += ps * nn.y * v_r[a];
        ga[2] += ps * nn.z * v_r[a];
        if (b >= 0) {
          double *gb = grad + ((size_t)b * ncomp + k) * 3;
          gb[0] -= ps * nn.x * v_r[b];
          gb[1] -= ps * nn.y * v_r[b];
          gb[2] -= ps * nn.z * v_r[b];
        }
      }
    }
    if (iter != n_iter) std::copy(grad, grad + G, g0.begin());
  }
  return 0;
}

int fvm_momentum_deferred(const fvm_mesh *m, int ncomp, const double *phi, const double *grad,
                          const double *flux, double mu, double c_bl, int scheme, double *rhs) {
  if (scheme < 0 || scheme > 3) return -1;
  const size_t F = m->f_ip.size();
  const double small = 1e-20;  // precision.f90:8
  auto aux = [](V3 xf, V3 nn, V3 xc) { return (xf - nn * dot(xf - xc, nn)) - xc; };
  for (size_t f = 0; f < F; ++f) {
    const int a = m->f_ip[f], b = m->f_in[f];
    if (b < 0) continue;
    double s, l, w;
    V3 nn, xf;
    m->face_geom(f, s, nn, xf, l, w);
    const V3 dxa = aux(xf, nn, m->xc[a]), dxb = aux(xf, nn, m->xc[b]);
    const double c = flux[f], d = mu * s / l;
    for (int k = 0; k < ncomp; ++k) {
      const double pa = phi[(size_t)a * ncomp + k], pb = phi[(size_t)b * ncomp + k];
      const double *ga = &grad[((size_t)a * ncomp + k) * 3];
      const double *gb = &grad[((size_t)b * ncomp + k) * 3];
      const double pa_aux = pa + dot({ga[0], ga[1], ga[2]}, dxa);
      const double pb_aux = pb + dot({gb[0], gb[1], gb[2]}, dxb);
      double cor = 0.0;
      if (c != 0.0) {
        double pf;
        if (scheme == 0) {
          pf = w * pb_aux + (1.0 - w) * pa_aux;
        } else {  // TVD (cfd_setup.f90:233-272)
          const bool fwd = c > 0.0;
          const double pc = fwd ? pa_aux : pb_aux, pd = fwd ? pb_aux : pa_aux;
          const double *gc = fwd ? ga : gb;
          const V3 xpa = m->xc[a] + dxa, xpb = m->xc[b] + dxb;
          const V3 dx = fwd ? xpb - xpa : xpa - xpb;
          const double pu = pd - 2.0 * dot({gc[0], gc[1], gc[2]}, dx);
          double r = (pc - pu) / (pd - pc + small);
          if (scheme == 1) r = std::max(0.0, std::min(1.0, r));
          else if (scheme == 2) r = (r + std::fabs(r)) / (1.0 + std::fabs(r) + small);
          else r = std::max({0.0, std::min(1.0, 2.0 * r), std::min(2.0, r)});
          pf = pc + 0.5 * r * (pd - pc);
        }
        const double up = c > 0.0 ? pa : pb;
        cor = c_bl * c * (up - pf);
      }
      cor = cor + d * ((pb_aux - pa_aux) - (pb - pa));
      rhs[(size_t)a * ncomp + k] += cor;
      rhs[(size_t)b * ncomp + k] -= cor;
    }
  }
  return 0;
}

namespace {
void face_flux(const fvm_mesh *m, const double *u, const double *p, const double *gradp,
               const double *ap, double rho, int aux_points, double *flux) {
  const size_t F = m->f_ip.size();
  auto aux = [](V3 xf, V3 nn, V3 xc) { return (xf - nn * dot(xf - xc, nn)) - xc; };
  std::vector<double> vol(m->n_cell);
  fvm_mesh_cell_geom(m, nullptr, vol.data());
  for (size_t f = 0; f < F; ++f) {
    const int a = m->f_ip[f], b = m->f_in[f];
    if (b < 0) {
      flux[f] = 0.0;
      continue;
    }
    double s, l, w;
    V3 nn, x;
    m->face_geom(f, s, nn, x, l, w);
    V3 uf{w * u[3 * b] + (1 - w) * u[3 * a], w * u[3 * b + 1] + (1 - w) * u[3 * a + 1],
          w * u[3 * b + 2] + (1 - w) * u[3 * a + 2]};
    const double p_r = w / (ap[b] + 1e-20) + (1 - w) / (ap[a] + 1e-20);
    const double v = w * vol[b] + (1 - w) * vol[a];
    const double d = rho * p_r * s * v / l;
    V3 gf{w * gradp[3 * b] + (1 - w) * gradp[3 * a], w * gradp[3 * b + 1] + (1 - w) * gradp[3 * a + 1],
          w * gradp[3 * b + 2] + (1 - w) * gradp[3 * a + 2]};
    double pa = p[a], pb = p[b];
    if (aux_points) {  // cfd_setup.f90:611-614: p at the auxiliary points
      pa = pa + dot({gradp[3 * a], gradp[3 * a + 1], gradp[3 * a + 2]}, aux(x, nn, m->xc[a]));
      pb = pb + dot({gradp[3 * b], gradp[3 * b + 1], gradp[3 * b + 2]}, aux(x, nn, m->xc[b]));
    }
    const double dp = (pb - pa) - dot(gf, m->xc[b] - m->xc[a]);
    flux[f] = rho * s * dot(uf, nn) - d * dp;
  }
}
}  // namespace

void fvm_face_flux(const fvm_mesh *m, const double *u, const double *p, const double *gradp,
                   const double *ap, double rho, double *flux) {
  face_flux(m, u, p, gradp, ap, rho, 0, flux);
}

void fvm_face_flux_aux(const fvm_mesh *m, const double *u, const double *p, const double *gradp,
                       const double *ap, double rho, double *flux) {
  face_flux(m, u, p, gradp, ap, rho, 1, flux);
}

double fvm_mass_imbalance(const fvm_mesh *m, const double *flux, int pin, double *b) {
  const int N = m->n_cell;
  const size_t F = m->f_ip.size();
  for (int c = 0; c < N; ++c) b[c] = 0.0;
  for (size_t f = 0; f < F; ++f) {
    const int a = m->f_ip[f], n = m->f_in[f];
    if (n < 0) continue;
    b[a] -= flux[f];
    b[n] += flux[f];
  }
  if (pin > 0) b[pin - 1] = 0.0;
  double t = 0.0;
  for (int c = 0; c < N; ++c) t += std::fabs(b[c]);
  return t;
}

void fvm_simple_correct(const fvm_mesh *m, const double *pp, const double *gradpp,
                        const double *ap, double rho, double urf_p, double *u, double *p,
                        double *flux) {
  const int N = m->n_cell;
  const size_t F = m->f_ip.size();
  std::vector<double> vol(N);
  fvm_mesh_cell_geom(m, nullptr, vol.data());
  for (int c = 0; c < N; ++c) {
    p[c] += urf_p * pp[c];
    const double k = vol[c] / (ap[c] + 1e-20);
    for (int d = 0; d < 3; ++d) u[3 * c + d] -= k * gradpp[3 * c + d];
  }
  for (size_t f = 0; f < F; ++f) {
    const int a = m->f_ip[f], b = m->f_in[f];
    if (b < 0) continue;
    double s, l, w;
    V3 nn, x;
    m->face_geom(f, s, nn, x, l, w);
    const double p_r = w / (ap[b] + 1e-20) + (1 - w) / (ap[a] + 1e-20);
    const double v = w * vol[b] + (1 - w) * vol[a];
    flux[f] -= rho * p_r * s * v / l * (pp[b] - pp[a]);
  }
}

void fvm_uniform(uint64_t seed, int64_t count, double *out) {
  std::mt19937_64 rng(seed);
  for (int64_t i = 0; i < count; ++i)
    out[i] = (double)(rng() >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
}

}  // extern "C"
