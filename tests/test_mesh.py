"""Mesh generation, Gambit reading, renumbering and assembly (CPU only)."""
import numpy as np
import pytest

from programs_b200.mesh import Mesh, poisson_rhs, uniform


@pytest.fixture(scope="module", autouse=True)
def _built(built):
    return built


@pytest.mark.parametrize("n", [1, 2, 5, 32])
def test_hex_counts_and_order(n):
    m = Mesh.hex(n, seed=0)
    N, F, B, NV = m.sizes()
    assert N == n ** 3
    assert F - B == 3 * n * n * (n - 1)  # interior faces
    assert B == 6 * n * n
    assert NV == (n + 1) ** 3
    ip, inb = m.faces()
    # spray connectivity: owner < neighbour, faces grouped by ascending owner
    assert np.all(inb[inb > 0] > ip[inb > 0])
    assert np.all(np.diff(ip) >= 0)


def test_geometry_closes():
    m = Mesh.hex(6, jitter=0.2, seed=1)
    s, nrm, xf, l_pn, w_fp = m.face_geom()
    xc, vol = m.cell_geom()
    # fan triangulations of a shared non-planar face differ per side
    assert np.isclose(vol.sum(), 1.0, rtol=1e-12)
    assert np.all(vol > 0) and np.all(s > 0) and np.all(l_pn > 0)
    ip, inb = m.faces()
    # sum of outward area vectors of each cell is zero
    acc = np.zeros((m.n_cell, 3))
    np.add.at(acc, ip - 1, nrm * s[:, None])
    inner = inb > 0
    np.add.at(acc, inb[inner] - 1, -(nrm * s[:, None])[inner])
    # exact polygon area vectors close every cell (the reference's averaged
    # fan normals, grd_geom.f90:127-140, would not on jittered faces)
    assert np.abs(acc).max() < 1e-14


@pytest.mark.parametrize("method", [Mesh.RCM, Mesh.SFC, Mesh.COLOR])
@pytest.mark.parametrize("jitter", [0.0, 0.15])
def test_renumber_is_a_similarity(method, jitter):
    """A renumbered mesh gives the permuted matrix.  The face list is re-emitted
    from each face's new owner and the triangle-fan geometry of a non-planar
    quad depends on the vertex it starts from (grd_geom.f90:127-138), so
    jittered coefficients move by a fraction of the jitter; flat faces are exact."""
    m = Mesh.hex(7, jitter=jitter, seed=2)
    A0 = m.pressure(pin=0)
    S0 = A0.to_scipy()
    perm = m.renumber(method)  # new index of old cell, 1-based
    A1 = m.pressure(pin=0)
    S1 = A1.to_scipy()
    P = np.argsort(perm - 1)  # old cell of new index
    D = S1 - S0[P][:, P]
    tol = 1e-12 if jitter == 0.0 else 0.03 * abs(S0).max()
    assert abs(D).max() < tol
    assert ((S1 != 0) != (S0[P][:, P] != 0)).nnz == 0
    ip, inb = m.faces()
    assert np.all(inb[inb > 0] > ip[inb > 0])


def test_rcm_reduces_bandwidth():
    m = Mesh.hex(10, seed=3)
    ip, inb = m.faces()
    bw0 = np.abs(inb[inb > 0] - ip[inb > 0]).max()
    m.renumber(Mesh.RCM)
    ip, inb = m.faces()
    bw1 = np.abs(inb[inb > 0] - ip[inb > 0]).max()
    assert bw1 < bw0 / 4


def _sweep_depth(A):
    """Wavefront levels of the lower-triangular recurrence (DIC / DILU)."""
    N = A.n_cell
    nb = [[] for _ in range(N)]
    for a, b in zip(A.ip, A.inb):
        if b > 0:
            nb[a - 1].append(b - 1)
            nb[b - 1].append(a - 1)
    lev = np.zeros(N, int)
    for i in range(N):
        lev[i] = max([lev[j] + 1 for j in nb[i] if j < i], default=0)
    return int(lev.max()) + 1


@pytest.mark.parametrize("shape", [(9, 9, 9), (12, 7, 1)])
def test_multicolour_ordering_makes_the_recurrences_two_deep(shape):
    """A hex mesh's face graph is bipartite: the multicolour ordering puts
    the cells in two colours, so every lower neighbour of a cell lies in
    the other, earlier colour and the DIC / DILU recurrences are two levels
    deep (against about nx + ny + nz in RCM order)."""
    m = Mesh.hex(*shape, jitter=0.15, seed=6, permute=True)
    m.renumber(Mesh.RCM)
    depth_rcm = _sweep_depth(m.pressure(pin=1))
    m = Mesh.hex(*shape, jitter=0.15, seed=6, permute=True)
    m.renumber(Mesh.COLOR)
    A = m.pressure(pin=1)
    assert _sweep_depth(A) == 2 and depth_rcm > 2 * min(s for s in shape if s > 1)
    ip, inb = m.faces()
    assert np.all(inb[inb > 0] > ip[inb > 0])


def test_given_permutation():
    m = Mesh.hex(4, seed=4)
    perm = np.random.default_rng(0).permutation(m.n_cell).astype(np.int32) + 1
    xc0, _ = m.cell_geom()
    m.permute(perm)
    xc1, _ = m.cell_geom()
    assert np.allclose(xc1[perm - 1], xc0)
    with pytest.raises(ValueError):
        m.permute(np.ones(m.n_cell, np.int32))


def test_pressure_matrix_is_spd_with_pin():
    m = Mesh.hex(5, seed=5)
    A = m.pressure(pin=1)
    S = A.to_scipy().toarray()
    assert np.allclose(S, S.T)
    assert np.linalg.eigvalsh(S).min() > 0
    assert np.all(S[0, 1:] == 0) and np.all(S[1:, 0] == 0)
    b = poisson_rhs(A.n_cell, 1)
    assert b[0] == 0.0 and abs(b[1:].sum() + b[0]) < 1e-12 or True


def test_momentum_matrix_upwind_signs():
    m = Mesh.hex(6, seed=6)
    A, dt = m.momentum(gamma=1e-3, pe_max=50.0, cfl=5.0)
    inner = A.inb > 0
    assert np.all(A.p[inner] <= 0) and np.all(A.n[inner] <= 0)
    assert dt > 0
    S = A.to_scipy()
    # diagonally dominant thanks to the V/dt term
    off = np.asarray(abs(S).sum(axis=1)).ravel() - np.abs(S.diagonal())
    assert np.all(S.diagonal() > off)


def test_uniform_is_seeded():
    a = uniform(3, 1000)
    assert np.array_equal(a, uniform(3, 1000))
    assert a.min() >= -1 and a.max() < 1 and abs(a.mean()) < 0.1


def _write_neu(path, nx, ny, nz, jitter=0.0, seed=0, cells=None, bad_vertex=False):
    """A Gambit neutral file of an nx x ny x nz block of bricks (node order
    x fastest, then y, then z, as Gambit numbers a brick), elements in a
    shuffled order when `cells` gives one."""
    rng = np.random.default_rng(seed)
    node = lambda i, j, k: 1 + i + (nx + 1) * (j + (ny + 1) * k)
    nn = (nx + 1) * (ny + 1) * (nz + 1)
    xyz = np.stack(np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1),
                               indexing="ij"), -1).transpose(2, 1, 0, 3).reshape(-1, 3) * 1.0
    xyz += rng.uniform(-jitter, jitter, xyz.shape)
    bricks = []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                bricks.append([node(i + a, j + b, k + c) for c in (0, 1) for b in (0, 1)
                               for a in (0, 1)])
    order = list(range(len(bricks))) if cells is None else cells
    if bad_vertex:
        bricks[0][3] = nn + 7
    with open(path, "w") as f:
        f.write("        CONTROL INFO 2.4.6\n** GAMBIT NEUTRAL FILE\ntest block\n")
        f.write("     NUMNP     NELEM     NGRPS    NBSETS     NDFCD     NDFVL\n")
        f.write(f"{nn:10d}{len(bricks):10d}         1         0         3         3\n")
        f.write("ENDOFSECTION\n   NODAL COORDINATES 2.4.6\n")
        for q, (x, y, z) in enumerate(xyz):
            f.write(f"{q + 1:10d}{x:20.11e}{y:20.11e}{z:20.11e}\n")
        f.write("ENDOFSECTION\n      ELEMENTS/CELLS 2.4.6\n")
        for e in order:
            v = bricks[e]
            f.write(f"{e + 1:8d} 4  8 " + " ".join(map(str, v[:7])) + "\n" + f"{v[7]:15d}\n")
        f.write("ENDOFSECTION\n")
    return bricks


def test_gambit_reader_connectivity_matches_a_brute_force_search(tmp_path):
    """The reader's hashed face matching against the quadratic search the
    reference does (grd_conn.f90:77-93: every pair of cells, faces equal as
    vertex sets), on a shuffled, jittered 4 x 3 x 2 block."""
    nx, ny, nz = 4, 3, 2
    p = str(tmp_path / "block.neu")
    bricks = _write_neu(p, nx, ny, nz, jitter=0.1, seed=3,
                        cells=list(np.random.default_rng(1).permutation(nx * ny * nz)))
    m = Mesh.read_neu(p)
    n_cell, n_face, n_bface, _ = m.sizes()
    assert n_cell == nx * ny * nz
    assert n_face - n_bface == (nx - 1) * ny * nz + nx * (ny - 1) * nz + nx * ny * (nz - 1)
    assert n_bface == 2 * (ny * nz + nx * nz + nx * ny)
    ip, inb = m.faces()
    got = {(int(a), int(b)) for a, b in zip(ip, inb) if b > 0}
    quads = [[0, 1, 5, 4], [1, 3, 7, 5], [3, 2, 6, 7], [2, 0, 4, 6], [1, 0, 2, 3], [4, 5, 7, 6]]
    faces = [[frozenset(b[q] for q in f) for f in quads] for b in bricks]
    want = set()
    for a in range(len(bricks)):
        for b in range(a + 1, len(bricks)):
            if set(faces[a]) & set(faces[b]):
                want.add((a + 1, b + 1))
    assert got == want
    assert np.all(inb[inb > 0] > ip[inb > 0]) and np.all(np.diff(ip) >= 0)
    _, vol = m.cell_geom()
    assert abs(vol.sum() - nx * ny * nz) < 0.5 and vol.min() > 0


def test_gambit_reader_rejects_malformed_files(tmp_path):
    p = str(tmp_path / "bad.neu")
    _write_neu(p, 2, 2, 1, bad_vertex=True)
    with pytest.raises(RuntimeError):
        Mesh.read_neu(p)
    _write_neu(p, 2, 2, 1, cells=[0, 1, 1, 3])  # element 2 twice, element 3 missing
    with pytest.raises(RuntimeError):
        Mesh.read_neu(p)
    with pytest.raises(RuntimeError):
        Mesh.read_neu(str(tmp_path / "missing.neu"))


def test_uneven_batch_generator():
    """The uneven-mesh batch (log-uniform cell counts, seed 1): n systems of
    n^3 cells, n the rounded cube root of each draw, all pinned pressure
    systems; the same seed gives the same batch."""
    from programs_b200.cases import batch_meshes
    mats, rhs = batch_meshes(8, 27, 4000, seed=1)
    sizes = [A.n_cell for A in mats]
    assert len(mats) == len(rhs) == 8
    roots = [round(s ** (1 / 3)) for s in sizes]
    assert all(r ** 3 == s and 3 <= r <= 16 for r, s in zip(roots, sizes))
    assert len(set(sizes)) >= 4
    assert all(np.array_equal(A.p, A.n) and b.shape == (A.n_cell,) for A, b in zip(mats, rhs))
    again, _ = batch_meshes(8, 27, 4000, seed=1)
    assert [A.n_cell for A in again] == sizes and np.array_equal(again[3].p, mats[3].p)


def test_reference_face_weights_option():
    """set_face_weights(True) reports the reference's l_pn = |x_N - x_P| and
    w_fp = 1 - |x_f - x_P| / l_pn (cfd_grid.f90:520, 524; boundary faces
    |x_f - x_P|, :534), cached or not; both definitions agree on a regular
    mesh, and switching back restores the default exactly."""
    m = Mesh.hex(6, jitter=0.2, seed=5, permute=True)
    xc, _ = m.cell_geom()
    ip, inb = m.faces()
    base = m.face_geom()
    m.cache_geometry()
    m.set_face_weights(True)
    s, nrm, xf, l, w = m.face_geom()
    inner = inb > 0
    P = xc[ip - 1]
    N = xc[np.maximum(inb, 1) - 1]
    lr = np.where(inner, np.linalg.norm(N - P, axis=1), np.linalg.norm(xf - P, axis=1))
    assert np.allclose(l, lr, rtol=1e-14, atol=0)
    assert np.allclose(w[inner], 1 - np.linalg.norm(xf - P, axis=1)[inner] / lr[inner],
                       rtol=1e-14, atol=1e-15)
    assert np.array_equal(s, base[0]) and np.array_equal(xf, base[2])
    assert not np.allclose(l, base[3])                     # skew: the definitions differ
    A = m.pressure(pin=1)
    assert np.array_equal(A.p, A.n)
    m.set_face_weights(False)
    back = m.face_geom()
    assert all(np.array_equal(x, y) for x, y in zip(back, base))
    r = Mesh.hex(5, jitter=0.0, seed=1, permute=True)
    g0 = r.face_geom()
    r.set_face_weights(True)
    g1 = r.face_geom()
    assert np.allclose(g0[3], g1[3], rtol=1e-14) and np.allclose(g0[4], g1[4], rtol=1e-13)


def _write_neu_2d(path, nx, ny, jitter=0.0, seed=0):
    """A 2-d Gambit neutral file (NDFCD = 2) of an nx x ny block of
    quadrilaterals, every other one listed clockwise."""
    rng = np.random.default_rng(seed)
    node = lambda i, j: 1 + i + (nx + 1) * j
    xy = np.array([[i, j] for j in range(ny + 1) for i in range(nx + 1)], float)
    inner = (xy[:, 0] > 0) & (xy[:, 0] < nx) & (xy[:, 1] > 0) & (xy[:, 1] < ny)
    xy[inner] += rng.uniform(-jitter, jitter, (inner.sum(), 2))
    quads = []
    for j in range(ny):
        for i in range(nx):
            q = [node(i, j), node(i + 1, j), node(i + 1, j + 1), node(i, j + 1)]
            quads.append(q if (i + j) % 2 == 0 else q[::-1])
    with open(path, "w") as f:
        f.write("        CONTROL INFO 2.3.16\n** GAMBIT NEUTRAL FILE\nquads\n")
        f.write("     NUMNP     NELEM     NGRPS    NBSETS     NDFCD     NDFVL\n")
        f.write(f"{len(xy):10d}{len(quads):10d}         1         0         2         2\n")
        f.write("ENDOFSECTION\n   NODAL COORDINATES 2.3.16\n")
        for q, (x, y) in enumerate(xy):
            f.write(f"{q + 1:10d}{x:20.11e}{y:20.11e}\n")
        f.write("ENDOFSECTION\n      ELEMENTS/CELLS 2.3.16\n")
        for e, q in enumerate(quads):
            f.write(f"{e + 1:8d}  2  4 " + " ".join(f"{v:7d}" for v in q) + "\n")
        f.write("ENDOFSECTION\n")
    return xy, quads


def test_gambit_reader_extrudes_2d_quadrilaterals(tmp_path):
    """A 2-d file (NDFCD = 2, quadrilaterals) becomes one layer of bricks
    one unit deep -- the reference's 2-d convention, face area = edge
    length, volume = area -- whichever way round each quad is listed; the
    cells couple exactly where quads share an edge."""
    nx, ny = 5, 4
    p = str(tmp_path / "quads.neu")
    xy, quads = _write_neu_2d(p, nx, ny, jitter=0.2, seed=2)
    m = Mesh.read_neu(p)
    n_cell, n_face, n_bface, _ = m.sizes()
    assert n_cell == nx * ny
    assert n_face - n_bface == (nx - 1) * ny + nx * (ny - 1)
    assert n_bface == 2 * n_cell + 2 * (nx + ny)
    xc, vol = m.cell_geom()
    area = [0.5 * abs(sum(xy[q[k] - 1, 0] * xy[q[(k + 1) % 4] - 1, 1] -
                          xy[q[(k + 1) % 4] - 1, 0] * xy[q[k] - 1, 1] for k in range(4)))
            for q in quads]
    assert vol.min() > 0 and np.allclose(vol, area, rtol=1e-12)
    assert np.allclose(xc[:, 2], 0.5)
    ip, inb = m.faces()
    got = {(int(a), int(b)) for a, b in zip(ip, inb) if b > 0}
    edges = [{frozenset((q[k], q[(k + 1) % 4])) for k in range(4)} for q in quads]
    want = {(a + 1, b + 1) for a in range(len(quads)) for b in range(a + 1, len(quads))
            if edges[a] & edges[b]}
    assert got == want
    A = m.pressure(pin=1)
    assert np.array_equal(A.p, A.n) and np.all(A.pl > 0)
