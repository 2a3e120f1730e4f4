"""Training and use of the learned preconditioner (the network in
programs_b200/csrc/gnn.cuh, applied by solv_gpu_fcg).

Training data are the pressure-correction systems the SIMPLE loop itself
generates (spray-simulation/cfd_setup.f90:604-646: d = rho (V/a_P)_f
area/l_pn, a_P the momentum diagonal of the current velocity field) on
jittered hex meshes of a lid-driven cavity, jitter uniform in [0, 0.25],
lid velocity in [0.1, 2]: the device-resident loop runs with the
reference's own solver settings and every outer iteration contributes its
matrix and mass-imbalance right-hand side (every other one a uniform random
right-hand side instead, so that both kinds are seen); each system several
residuals, taken from the Jacobi-PCG iterates the plain solver visits.  The losses need no reference solutions: with z the
preconditioned residual, the energy J = 1/2 z'Az - z'r (loss 0, minimised
by z = A^-1 r) or the scale-free -(z'r)^2/(z'Az) (the energy after the
best step along z, which is what one CG step takes, free in the overall
scale of z as flexible CG is), for z = K r with the network's operator K
alone (losses 0 and 1) or, as -log((z'r)^2/(z'Az)) so that every sample
counts alike, for z = V(r), the V-cycle of the aggregation hierarchy with
K as its finest-level smoother (loss 2, the default: the preconditioner
solv_gpu_fcg applies), differentiated through the V-cycle.  Forward,
backward and the Adam step run on the GPU in the library's own kernels;
this module only orchestrates.

  python -m programs_b200.learn --size 64 --meshes 40 --per-mesh 50 --out weights.npz
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from .mesh import Mesh, cavity_field, momentum_field, poisson_rhs, pressure_correction
from .solver import BAD_INPUT, GpuSolver, SolverError

H, NF, NL = 32, 4, 3
P_WIN = 0
P_LAYER = H * NF
LAYER_SZ = 2 * H * H + H
P_WA = P_LAYER + NL * LAYER_SZ  # diagonal-scale head
P_BA = P_WA + H
P_WE = P_BA + 1                 # face head
P_BE = P_WE + H
N_PARAM = P_BE + 1
LAYOUT = "H32-NF4-NL3-spd-v2"

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "weights", "gnn_pressure.npz")


def init_params(seed: int = 0) -> np.ndarray:
    """Random hidden layers, zero heads: the untrained preconditioner is the
    Jacobi step (s = sqrt(softplus(0)/softplus(0)) = 1, E = 0)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAM, np.float32)
    p[P_WIN:P_WIN + H * NF] = rng.normal(0, 0.5, H * NF)
    for l in range(NL):
        o = P_LAYER + l * LAYER_SZ
        p[o:o + H * H] = rng.normal(0, 0.3 / np.sqrt(H), H * H)            # Ws
        p[o + H * H:o + 2 * H * H] = rng.normal(0, 0.3 / np.sqrt(H), H * H)  # Wn
    return p


def save_params(path: str, p: np.ndarray, meta: dict) -> None:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez(path, params=np.asarray(p, np.float32), n_param=N_PARAM, layout=LAYOUT,
             meta=json.dumps(meta))


def load_params(path: str = DEFAULT_WEIGHTS) -> np.ndarray:
    d = np.load(path)
    if int(d["n_param"]) != N_PARAM or str(d["layout"]) != LAYOUT:
        raise ValueError(f"{path}: parameter layout does not match this library's network")
    return np.asarray(d["params"], np.float32)


def simple_systems(size: int, n_mesh: int, per_mesh: int, seed: int = 0):
    """Yield (mesh, pressure-correction FaceMatrix, rhs) as the SIMPLE loop
    would assemble them: per mesh, per_mesh flow states (lid velocity,
    flow development)."""
    rng = np.random.default_rng(seed)
    for k in range(n_mesh):
        jit = float(rng.uniform(0.0, 0.25))
        m = Mesh.hex(size, jitter=jit, seed=seed * 1000 + k, permute=True)
        m.renumber(Mesh.RCM)
        m.cache_geometry()
        for j in range(per_mesh):
            lid = float(np.exp(rng.uniform(np.log(0.1), np.log(2.0))))
            # flow development within the outer loop: scale of the field
            dev = float(rng.uniform(0.2, 1.0))
            u = cavity_field(m, lid * dev)
            M, _, _ = momentum_field(m, u, u_lid=lid, mu=1e-3, urf=0.7)
            P = pressure_correction(m, M.pl, pin=1)
            b = poisson_rhs(P.n_cell, seed * 100000 + k * 1000 + j)
            yield m, P, b


def device_systems(size: int, n_mesh: int, per_mesh: int, seed: int = 0, device: int = 0,
                   stream=None):
    """The systems of simple_systems (same draws, same values bit for bit),
    assembled on the GPU (programs_b200.fv): yields (mesh, structure-only
    FaceMatrix of the first system of each mesh or None, (p, n, pl) device
    tensors, rhs)."""
    import torch

    from .fv import GpuFv
    from .mesh import FaceMatrix
    rng = np.random.default_rng(seed)
    dev = torch.device("cuda", device)
    for k in range(n_mesh):
        jit = float(rng.uniform(0.0, 0.25))
        m = Mesh.hex(size, jitter=jit, seed=seed * 1000 + k, permute=True)
        m.renumber(Mesh.RCM)
        m.cache_geometry()
        fv = GpuFv(m, device)
        if stream is not None:
            fv._lib.fv_gpu_set_stream(fv._h, stream.cuda_stream)
        ip, inb = m.faces()
        shell = FaceMatrix(m.n_cell, ip, inb, np.zeros(ip.shape[0]), np.zeros(ip.shape[0]),
                           np.ones(m.n_cell))
        for j in range(per_mesh):
            lid = float(np.exp(rng.uniform(np.log(0.1), np.log(2.0))))
            dev_scale = float(rng.uniform(0.2, 1.0))
            u = torch.from_numpy(cavity_field(m, lid * dev_scale)).to(dev)
            _, _, pl_m, _, _ = fv.momentum_field(u, None, rho=1.0, mu=1e-3, u_lid=lid, urf=0.7)
            pcn = fv.pressure_correction(pl_m, rho=1.0, pin=1)
            b = poisson_rhs(m.n_cell, seed * 100000 + k * 1000 + j)
            yield m, (shell if j == 0 else None), pcn, b
        fv.close()


def loop_systems(size: int, n_mesh: int, per_mesh: int, seed: int = 0, device: int = 0,
                 stream=None):
    """Pressure-correction systems as the SIMPLE loop generates them: per
    mesh (jitter uniform in [0, 0.25]) and lid velocity (log-uniform in
    [0.1, 2], mu = 1e-3), per_mesh outer iterations of the device-resident
    loop with the reference's own solver settings (momentum BiCGSTAB + DILU
    to 0.1 in at most 5 iterations, pressure DIC-PCG to 0.1 in at most 20,
    cfd_setup.f90:61,528,580,662).  Yields, at every outer iteration,
    (structure-only FaceMatrix of a new mesh or None, (p, n, pl) device
    tensors of the pressure-correction matrix, its right-hand side -- the
    mass imbalance -- as a device tensor)."""
    import torch

    from .fv import GpuFv
    from .mesh import FaceMatrix
    rng = np.random.default_rng(seed)
    dev = torch.device("cuda", device)
    rho, mu = 1.0, 1e-3
    for k in range(n_mesh):
        jit = float(rng.uniform(0.0, 0.25))
        lid = float(np.exp(rng.uniform(np.log(0.1), np.log(2.0))))
        m = Mesh.hex(size, jitter=jit, seed=seed * 1000 + k, permute=True)
        m.renumber(Mesh.RCM)
        m.cache_geometry()
        N = m.n_cell
        fv = GpuFv(m, device)
        sm, sp = GpuSolver(device), GpuSolver(device)
        if stream is not None:
            fv._lib.fv_gpu_set_stream(fv._h, stream.cuda_stream)
            sm.set_stream(stream.cuda_stream)
            sp.set_stream(stream.cuda_stream)
        ip, inb = m.faces()
        shell = FaceMatrix(N, ip, inb, np.zeros(ip.shape[0]), np.zeros(ip.shape[0]), np.ones(N))
        sm.matrix_set(shell)
        sp.matrix_set(shell)
        _, vol_h = m.cell_geom()
        vol = torch.from_numpy(vol_h).to(dev)
        u = torch.zeros(N, 3, dtype=torch.float64, device=dev)
        p = torch.zeros(N, dtype=torch.float64, device=dev)
        F = None
        for j in range(per_mesh):
            gradp = fv.gradient(p)
            Mp, Mn, Mpl, rhs, Fm = fv.momentum_field(u, flux=F, rho=rho, mu=mu, u_lid=lid, urf=0.7)
            if F is None:
                F = Fm
            rhs -= gradp * vol[:, None]
            sm.matrix_values_dev(Mp.data_ptr(), Mn.data_ptr(), Mpl.data_ptr())
            res0 = rhs.t().contiguous()
            sm.solv_bicg_dev(2, 0.1, 5, 3, u.data_ptr(), res0.data_ptr())
            F = fv.face_flux(u, p, gradp, Mpl, rho)
            Pp, Pn, Ppl = fv.pressure_correction(Mpl, rho=rho, pin=1)
            b, _ = fv.mass_imbalance(F, pin=1)
            yield (shell if j == 0 else None), (Pp, Pn, Ppl), b.clone()
            sp.matrix_values_dev(Pp.data_ptr(), Pn.data_ptr(), Ppl.data_ptr())
            pp = torch.zeros(N, dtype=torch.float64, device=dev)
            sp.solv_cg_dev(1, 0.1, 20, 1, pp.data_ptr(), b.data_ptr(), not_r0=True)
            fv.simple_correct(pp, fv.gradient(pp), Mpl, rho, 0.3, u, p, F)
        sm.close()
        sp.close()
        fv.close()


def _residual_samples(s: GpuSolver, b_dev, n_samples, rng, torch, max_k=400):
    """[b, r_k1, r_k2, ...]: residuals b - A x_k of Jacobi-PCG after k
    iterations (the residuals the solver visits), as one (n, N) tensor."""
    N = b_dev.shape[0]
    phi = torch.zeros(N, dtype=torch.float64, device=b_dev.device)
    res0 = torch.empty_like(b_dev)
    y = torch.empty_like(b_dev)
    out = torch.empty((n_samples, N), dtype=torch.float64, device=b_dev.device)
    out[0].copy_(b_dev)
    ks = sorted(np.exp(rng.uniform(0, np.log(max_k), n_samples - 1)).astype(int).tolist())
    for m, k in enumerate(ks, start=1):
        phi.zero_()
        res0.copy_(b_dev)
        s.solv_cg_dev(0, 1e-300, int(max(k, 1)), 1, phi.data_ptr(), res0.data_ptr())
        s.spmv_dev(phi.data_ptr(), y.data_ptr())
        out[m].copy_(b_dev - y)
    return out


def validation_loss(s: GpuSolver, systems, torch) -> float:
    """Mean loss of the current parameters over fixed held-out systems
    [(shell, (p, n, pl), b)], each with its right-hand side as the one
    sample: the same systems before and after training, so the two numbers
    compare (the running training loss mixes systems of different kinds)."""
    vals = []
    for shell, (p_d, n_d, pl_d), b_dev in systems:
        s.matrix_set(shell)
        s.matrix_values_dev(p_d.data_ptr(), n_d.data_ptr(), pl_d.data_ptr())
        vals.append(s.gnn_grad_dev(b_dev.data_ptr(), b_dev.data_ptr(), 1))
    s.gnn_zero_grad()
    return float(np.mean(vals))


def train(size=64, n_mesh=40, per_mesh=50, samples=4, epochs=1, lr=2e-3, seed=0,
          init=None, log_every=50, device=0, loss=2, smoother=1, data="synthetic", n_val=6):
    """smoother (loss 2): 1 trains the network's operator K as the V-cycle's
    smoother, 2 its per-cell diagonal alone (learned Jacobi weights).
    data: "synthetic" (the default, and what the shipped network was
    trained on) -- cavity-like flow states with random right-hand sides
    (device_systems); "loop" -- the systems the SIMPLE loop generates
    (loop_systems), every other one with a uniform random right-hand side
    in place of the mass imbalance, so that both kinds are seen."""
    import torch
    from .solver import OPT_GNN_LOSS, OPT_MG_SMOOTHER
    s = GpuSolver(device)
    s.set_option(OPT_GNN_LOSS, loss)
    s.set_option(OPT_MG_SMOOTHER, smoother)
    p = init_params(seed) if init is None else np.asarray(init, np.float32)
    s.gnn_set_params(p)
    rng = np.random.default_rng(seed + 7)
    dev = torch.device("cuda", device)
    # one stream for the library and for torch's element-wise work
    stream = torch.cuda.Stream(device=dev)
    s.set_stream(stream.cuda_stream)
    hist = []
    t0 = time.time()
    step = 0
    skipped = 0
    with torch.cuda.stream(stream):
        # held-out systems of the same kind (another seed), each kept whole
        val_sys = []
        if data == "loop":
            vgen = loop_systems(size, n_val, 1, seed=seed + 1000, device=device, stream=stream)
            for shell, (p_d, n_d, pl_d), b in vgen:
                val_sys.append((shell, (p_d.clone(), n_d.clone(), pl_d.clone()), b.clone()))
        else:
            for _, shell, (p_d, n_d, pl_d), b in device_systems(size, n_val, 1, seed=seed + 1000,
                                                                  device=device, stream=stream):
                val_sys.append((shell, (p_d.clone(), n_d.clone(), pl_d.clone()),
                                torch.from_numpy(b).to(dev)))
        val_before = validation_loss(s, val_sys, torch)
        for ep in range(epochs):
            if data == "loop":
                gen = loop_systems(size, n_mesh, per_mesh, seed=seed + ep, device=device,
                                   stream=stream)
            else:
                gen = ((shell, pcn, torch.from_numpy(b).to(dev)) for _, shell, pcn, b in
                       device_systems(size, n_mesh, per_mesh, seed=seed + ep, device=device,
                                      stream=stream))
            for shell, (p_d, n_d, pl_d), b_dev in gen:
                if shell is not None:
                    s.matrix_set(shell)  # structure of a new mesh
                s.matrix_values_dev(p_d.data_ptr(), n_d.data_ptr(), pl_d.data_ptr())
                if data == "loop" and step % 2 == 1:  # the other kind of right-hand side
                    b_dev = torch.from_numpy(poisson_rhs(b_dev.shape[0], seed * 7919 + step)).to(dev)
                rs = _residual_samples(s, b_dev, samples, rng, torch)
                try:
                    val = s.gnn_grad_dev(b_dev.data_ptr(), rs.data_ptr(), rs.shape[0])
                except SolverError as e:
                    # the multigrid loss on a system whose hierarchy could not
                    # be built (coarsening stalled): no gradient from it
                    if loss != 2 or e.code != BAD_INPUT:
                        raise
                    skipped += 1
                    continue
                s.gnn_adam(lr, 1.0)
                step += 1
                hist.append(val)
                if log_every and step % log_every == 0:
                    print(json.dumps({"step": step, "loss": float(np.mean(hist[-log_every:])),
                                      "t": round(time.time() - t0, 1)}), flush=True)
        val_after = validation_loss(s, val_sys, torch)
    stream.synchronize()
    p = s.gnn_get_params()
    s.close()
    return p, hist, {"val_loss_before": val_before, "val_loss_after": val_after,
                     "val_systems": len(val_sys), "skipped_systems": skipped}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=64)
    ap.add_argument("--meshes", type=int, default=40)
    ap.add_argument("--per-mesh", type=int, default=50)
    ap.add_argument("--samples", type=int, default=4)
    ap.add_argument("--epochs", type=int, default=1)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--resume", default=None)
    ap.add_argument("--loss", type=int, default=2,
                    help="0 energy, 1 scale-free (network alone), 2 scale-free through the V-cycle")
    ap.add_argument("--smoother", type=int, default=1,
                    help="loss 2: 1 the operator K, 2 its diagonal (learned Jacobi weights)")
    ap.add_argument("--data", default="synthetic", choices=["synthetic", "loop"],
                    help="synthetic: cavity-like flow states (the shipped network); "
                         "loop: the SIMPLE loop's own systems")
    ap.add_argument("--out", default="gnn_pressure_trained.npz",
                    help="where to write the weights; the shipped network is "
                         "programs_b200/weights/gnn_pressure.npz, replaced only when named")
    a = ap.parse_args(argv)
    init = load_params(a.resume) if a.resume else None
    t = time.time()
    p, hist, val = train(a.size, a.meshes, a.per_mesh, a.samples, a.epochs, a.lr, a.seed, init,
                         loss=a.loss, smoother=a.smoother, data=a.data)
    meta = {"size": a.size, "loss": a.loss, "smoother": a.smoother, "data": a.data,
            "systems": a.meshes * a.per_mesh * a.epochs, "samples": a.samples,
            "lr": a.lr, "seed": a.seed, "first_loss": float(np.mean(hist[:20])),
            "last_loss": float(np.mean(hist[-20:])), **val,
            "train_s": round(time.time() - t, 1)}
    save_params(a.out, p, meta)
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
