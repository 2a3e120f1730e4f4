"""CPU reference of the learned preconditioner's network and loss
(TEST INFRASTRUCTURE ONLY: the checker for programs_b200/csrc/gnn.cuh).

The reference code base has no learned preconditioner, so this is a
restatement of the network as specified in gnn.cuh, in float64 on the CPU,
with BF16 rounding emulated at exactly the points the GPU rounds (weights,
stored hidden states, aggregated messages) and straight-through gradients
there, as the GPU backward kernels use.  Gradients come from torch autograd
on the CPU, an implementation independent of the hand-written backward
kernels they check.
"""
from __future__ import annotations

import numpy as np
import torch

H, NF, NL = 32, 4, 3
P_WIN = 0
P_LAYER = H * NF
LAYER_SZ = 2 * H * H + H
P_WOUT = P_LAYER + NL * LAYER_SZ
P_C = P_WOUT + H
N_PARAM = P_C + 1


def bf16_round(x: torch.Tensor) -> torch.Tensor:
    """Round to the nearest BF16 (ties to even) through float32, as __float2bfloat16."""
    x32 = x.detach().to(torch.float32).contiguous()
    bits = x32.view(torch.int32).to(torch.int64) & 0xFFFFFFFF
    lsb = (bits >> 16) & 1
    r = ((bits + 0x7FFF + lsb) & 0xFFFF0000)
    r = torch.where(r >= 2 ** 31, r - 2 ** 32, r).to(torch.int32)
    return r.view(torch.float32).to(x.dtype)


ROUND = True  # False: exact float64 network (finite-difference checks)


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


def forward(A, r, params, grad=False):
    """z = M(r) and the per-cell energy loss J/N; returns (z, loss, params_tensor)."""
    rsd, frs, fdeg, rows, cols, w = features(A)
    N = A.n_cell
    r32 = np.asarray(r, np.float64).astype(np.float32)
    s = float(np.sum(np.abs(r32.astype(np.float64)) * rsd.astype(np.float64)) / N)
    inv_s = np.float32(1.0 / s)
    u = (r32 * rsd * inv_s).astype(np.float32)
    P = torch.tensor(np.asarray(params, np.float64), requires_grad=grad)
    ut = torch.tensor(u, dtype=torch.float64)
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
    out = bf(P[P_C]) * ut + h @ bf(P[P_WOUT:P_WOUT + H])
    aout = out - adj(out[:, None])[:, 0]
    J = (0.5 * out @ aout - out @ ut) / N
    z = out.detach().numpy() * s * rsd.astype(np.float64)
    return z, J, P


def loss_and_grad(A, r, params):
    _, J, P = forward(A, r, params, grad=True)
    J.backward()
    return float(J.detach()), P.grad.numpy().copy()
