"""CPU reference of the learned preconditioner (TEST INFRASTRUCTURE ONLY:
the oracle that programs_b200/csrc/gnn.cuh is tested against).

The reference code base has no learned preconditioner, so this restates
the network and preconditioner as specified in gnn.cuh, in float64 on the
CPU, with BF16 rounding emulated at exactly the points the GPU rounds
(weights, stored hidden states, aggregated messages) and straight-through
gradients there, as the GPU backward kernels use.  Gradients come from
torch autograd on the CPU, an implementation independent of the
hand-written backward kernels they check.
"""
from __future__ import annotations

import numpy as np
import torch

H, NF, NL = 32, 4, 3
P_WIN = 0
P_LAYER = H * NF
LAYER_SZ = 2 * H * H + H
P_WA = P_LAYER + NL * LAYER_SZ
P_BA = P_WA + H
P_WE = P_BA + 1
P_BE = P_WE + H
N_PARAM = P_BE + 1
GAMMA = 0.95

ROUND = True  # False: exact float64 network (finite-difference checks)


def bf16_round(x: torch.Tensor) -> torch.Tensor:
    """Round to the nearest BF16 (ties to even) through float32, as __float2bfloat16."""
    x32 = x.detach().to(torch.float32).contiguous()
    bits = x32.view(torch.int32).to(torch.int64) & 0xFFFFFFFF
    lsb = (bits >> 16) & 1
    r = ((bits + 0x7FFF + lsb) & 0xFFFF0000)
    r = torch.where(r >= 2 ** 31, r - 2 ** 32, r).to(torch.int32)
    return r.view(torch.float32).to(x.dtype)


def bf(x: torch.Tensor) -> torch.Tensor:
    """BF16 rounding with a straight-through gradient."""
    if not ROUND:
        return x
    return x + (bf16_round(x) - x).detach()


def features(A):
    """rsd, frs, fdeg (float32 as stored on the GPU) and the edge list."""
    N = A.n_cell
    d = np.asarray(A.pl, np.float64)
    rsd = 1.0 / np.sqrt(d)
    m = A.inb > 0
    a = A.ip[m] - 1
    b = A.inb[m] - 1
    rows = np.concatenate([a, b])
    cols = np.concatenate([b, a])
    vals = np.concatenate([A.p[m], A.n[m]])
    rs = np.zeros(N)
    np.add.at(rs, rows, vals)
    deg = np.zeros(N)
    np.add.at(deg, rows, 1.0)
    w = (-vals * rsd[rows] * rsd[cols]).astype(np.float32)
    return (rsd.astype(np.float32), (rs / d).astype(np.float32), (deg / 6.0).astype(np.float32),
            rows, cols, w)


def _scaled(r, rsd):
    """u = r rsd / s (float32 as the GPU), s = mean |r| rsd."""
    r32 = np.asarray(r, np.float64).astype(np.float32)
    s = float(np.sum(np.abs(r32.astype(np.float64)) * rsd.astype(np.float64)) / r32.shape[0])
    return (r32 * rsd * np.float32(1.0 / s)).astype(np.float32), s


def build(A, r0, params, grad=False):
    """The preconditioner the network builds from r0: (s, gE per directed
    edge, edge arrays, params tensor, features)."""
    rsd, frs, fdeg, rows, cols, w = features(A)
    N = A.n_cell
    u0, _ = _scaled(r0, rsd)
    P = torch.tensor(np.asarray(params, np.float64), requires_grad=grad)
    ut = torch.tensor(u0, dtype=torch.float64)
    x = torch.stack([ut, torch.tensor(frs, dtype=torch.float64),
                     torch.tensor(fdeg, dtype=torch.float64), torch.ones(N, dtype=torch.float64)], 1)
    rows_t, cols_t = torch.tensor(rows), torch.tensor(cols)
    wt = torch.tensor(w, dtype=torch.float64)

    def adj(h):  # agg_i = sum_j w_ij h_j
        out = torch.zeros_like(h)
        out.index_add_(0, rows_t, wt[:, None] * h[cols_t])
        return out

    Win = bf(P[P_WIN:P_WIN + H * NF].reshape(H, NF))
    h = bf(torch.relu(x @ Win.T))
    for l in range(NL):
        o = P_LAYER + l * LAYER_SZ
        Ws = bf(P[o:o + H * H].reshape(H, H))
        Wn = bf(P[o + H * H:o + 2 * H * H].reshape(H, H))
        b = bf(P[o + 2 * H * H:o + 2 * H * H + H])
        agg = bf(adj(h))
        pre = h @ Ws.T + agg @ Wn.T + b
        h = bf(h + torch.relu(pre))
    pa = h @ bf(P[P_WA:P_WA + H]) + bf(P[P_BA])
    s = torch.sqrt(torch.nn.functional.softplus(pa) / np.log(2.0))
    he = h @ bf(P[P_WE:P_WE + H])
    pre_e = 0.5 * (he[rows_t] + he[cols_t]) + bf(P[P_BE])
    gE = GAMMA * torch.tanh(pre_e) * wt
    return s, gE, rows_t, cols_t, wt, P, rsd


def _apply(q, gE, rows_t, cols_t, v):
    """q (v q + E (q v)) with E given per directed edge."""
    y = q * v
    t = y.clone()
    t.index_add_(0, rows_t, gE * y[cols_t])
    return q * t


def precondition(A, r0, r, params):
    """z = M^-1 r in the caller's space (float64 result)."""
    s, gE, rows_t, cols_t, wt, _, rsd = build(A, r0, params)
    q = s.detach() * torch.tensor(rsd, dtype=torch.float64)
    rt = torch.tensor(np.asarray(r, np.float64).astype(np.float32), dtype=torch.float64)
    return _apply(q, gE.detach(), rows_t, cols_t, rt).numpy()


def loss(A, r0, samples, params, grad=False, kind=1):
    """Mean over samples of L/N with z = K u (scaled space):
    kind 0: L = 1/2 z.Â z - z.u (energy of z);
    kind 1: L = -(z.u)^2 / (z.Â z) (energy after the best step along z)."""
    s, gE, rows_t, cols_t, wt, P, rsd = build(A, r0, params, grad=grad)
    N = A.n_cell
    J = 0.0
    for r in samples:
        u, _ = _scaled(r, rsd)
        ut = torch.tensor(u, dtype=torch.float64)
        z = _apply(s, gE, rows_t, cols_t, ut)
        az = z.clone()
        az.index_add_(0, rows_t, -wt * z[cols_t])
        if kind == 0:
            J = J + (0.5 * z @ az - z @ ut) / N
        else:
            J = J - (z @ ut) ** 2 / (z @ az) / N
    return J / len(samples), P


def loss_and_grad(A, r0, samples, params, kind=1):
    J, P = loss(A, r0, samples, params, grad=True, kind=kind)
    J.backward()
    return float(J.detach()), P.grad.numpy().copy()


def _sparse(M):
    M = M.tocoo()
    idx = torch.tensor(np.vstack([M.row, M.col]), dtype=torch.int64)
    return torch.sparse_coo_tensor(idx, torch.tensor(M.data, dtype=torch.float64), M.shape,
                                   check_invariants=True).coalesce()


def hierarchy(A, aggs):
    """Galerkin levels A_{l+1} = P_l^T A_l P_l of the piecewise-constant
    prolongations given by aggs[l] (level-l cell -> level-(l+1) aggregate)."""
    import scipy.sparse as sp
    mats, Ps = [A.to_scipy().tocsr()], []
    for a in aggs:
        a = np.asarray(a)
        P = sp.csr_matrix((np.ones(len(a)), (np.arange(len(a)), a)), shape=(len(a), int(a.max()) + 1))
        Ps.append(P)
        mats.append((P.T @ mats[-1] @ P).tocsr())
    return mats, Ps


def vcycle(mats, Ps, b, smooth0, omega, alpha, l=0):
    """One symmetric V-cycle on level l: w S b pre-smoothing from zero,
    coarse correction scaled by alpha, w S post-smoothing; S = smooth0 on
    level 0, D^-1 below; the coarsest level solved exactly (torch, float64)."""
    A = mats[l]
    if l == len(mats) - 1:
        return torch.linalg.solve(torch.tensor(A.toarray()), b)
    At = _sparse(A)
    if l == 0:
        S = smooth0
    else:
        dinv = torch.tensor(1.0 / A.diagonal())
        S = lambda v: dinv * v
    mv = lambda v: torch.sparse.mm(At, v[:, None])[:, 0]
    Pt = _sparse(Ps[l])
    x = omega * S(b)
    t = b - mv(x)
    xc = vcycle(mats, Ps, torch.sparse.mm(Pt.t(), t[:, None])[:, 0], smooth0, omega, alpha, l + 1)
    x = x + alpha * torch.sparse.mm(Pt, xc[:, None])[:, 0]
    return x + omega * S(b - mv(x))


def loss_mg(A, r0, samples, params, aggs, omega, alpha, grad=False, diag=False):
    """Mean over samples of L/N, L = -log((z.b)^2/(z.A z)) with z the
    V-cycle applied to b = r / gs, the network's operator
    K = D^-1/2 S (I+E) S D^-1/2 smoothing level 0 (the loss the GPU trains
    with through the V-cycle)."""
    s, gE, rows_t, cols_t, wt, P, rsd = build(A, r0, params, grad=grad)
    if diag:  # smoother 2: the per-cell scales alone (learned Jacobi weights)
        gE = gE * 0.0
    rsd_t = torch.tensor(rsd, dtype=torch.float64)
    K = lambda v: rsd_t * _apply(s, gE, rows_t, cols_t, rsd_t * v)
    mats, Ps = hierarchy(A, aggs)
    At = _sparse(mats[0])
    N = A.n_cell
    J = 0.0
    for r in samples:
        _, gs = _scaled(r, rsd)
        b = torch.tensor(np.asarray(r, np.float64).astype(np.float32).astype(np.float64) / gs,
                         dtype=torch.float64)
        z = vcycle(mats, Ps, b, K, omega, alpha)
        az = torch.sparse.mm(At, z[:, None])[:, 0]
        J = J - torch.log((z @ b) ** 2 / (z @ az)) / N
    return J / len(samples), P


def loss_mg_and_grad(A, r0, samples, params, aggs, omega, alpha, diag=False):
    J, P = loss_mg(A, r0, samples, params, aggs, omega, alpha, grad=True, diag=diag)
    J.backward()
    return float(J.detach()), P.grad.numpy().copy()
