"""SIMPLE outer loop for the 3-D lid-driven cavity, with the linear solves
on the GPU through the C-ABI -- the split the reference has, assembly on
the host (spray-simulation/cfd_solve.f90:131-179 calling cfd_setup_eqn and
cfd_setup_pp) and the solver swapped for the B200 one.

Per outer iteration:
  grad p (Green-Gauss)                              solv_grad, cfd_setup.f90:765
  momentum: upwind + diffusion, -grad p V, urf_u    cfd_setup.f90:178-518
  u* = solve (BiCGSTAB + DILU, u, v, w in one call) cfd_setup.f90:528
  face flux with Rhie-Chow pressure smoothing       cfd_setup.f90:615-634
  pressure correction: d = rho (V/a_P)_f area/l_pn  cfd_setup.f90:604-646
  p' = solve (CG, or FCG with the learned preconditioner)   :662
  p += urf_p p', u -= V/a_P grad p', F -= d dp'     cfd_setup.f90:689-729

  python -m programs_b200.simple --size 32 --outer 200 [--learned] [--device-assembly]

With --device-assembly (run_device) every piece above runs on the GPU
(programs_b200/fv.py, include/fv_gpu.h), bit-for-bit as on the host.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from .mesh import (Mesh, face_flux, gradient, gradient_sweeps, mass_imbalance,
                   momentum_deferred, momentum_field, pressure_correction, simple_correct)
from .solver import GpuSolver, OPT_FCG_FALLBACK, OPT_FCG_RELIABLE_DELTA, OPT_PRECISION


def run(size=32, n_outer=200, re=1000.0, u_lid=1.0, urf_u=0.7, urf_p=0.3, jitter=0.15, seed=0,
        p_reduc=1e-10, p_iter=20000, m_reduc=0.1, m_iter=5, learned=None, p_imat=1,
        m_precision=0, device=0, log_every=0, make_solver=None, reference_terms=False,
        reference_weights=False, p_scale=False):
    """Returns (u (N,3), p (N,), history, timings).  learned: weights array
    (FCG with the learned preconditioner for the pressure correction) or
    None (plain FP64 PCG with imat p_imat).  make_solver(device) builds the
    two solver contexts (default GpuSolver); anything with the same
    matrix_set / matrix_values / solv_cg / solv_bicg / set_option / close
    methods can stand in.  reference_terms adds what the reference's
    assembly has beyond the implicit terms: gradients by n_grad = 2
    corrected sweeps (cfd_solve.f90:38) with the velocity's wall values
    (neu = 0, cfd_setup.f90:124) and extrapolated pressure walls (neu = 2,
    :689, 754), and the explicit momentum terms (central deferred
    correction, non-orthogonal diffusion correction, :185-328) and the
    pressures at the auxiliary points in the face fluxes (:611-620).
    run_device does the same on the GPU.  reference_weights takes the
    reference's face distance and interpolation weight
    (Mesh.set_face_weights).  p_scale multiplies each pressure-correction
    right-hand side by the power of two nearest n_cell / sum|b| before the
    solve and divides the solution by it after: exact in floating point, so
    the solvers' arithmetic is unchanged except that the reference's
    absolute guard 1e-20 on the CG step (solv_cg.f90:67-68) acts on numbers
    of order one instead of the shrinking mass imbalance."""
    rho = 1.0
    mu = rho * u_lid * 1.0 / re
    m = Mesh.hex(size, jitter=jitter, seed=seed, permute=True)
    m.renumber(Mesh.RCM)
    if reference_weights:
        m.set_face_weights(True)
    m.cache_geometry()
    N = m.n_cell
    _, vol = m.cell_geom()
    u = np.zeros((N, 3))
    p = np.zeros(N)
    F = None
    if reference_terms:
        _, nrm, xf, _, _ = m.face_geom()
        _, inb = m.faces()
        wall_u = np.zeros((m.n_face, 3))  # no-slip walls, the y = 1 lid moving
        wall_u[(inb == 0) & (nrm[:, 1] > 0.9) & (xf[:, 1] > 1.0 - 1e-9), 0] = u_lid
        grad_p = lambda q: gradient_sweeps(m, q, 2, 2)
    else:
        grad_p = lambda q: gradient(m, q)
    factory = make_solver or GpuSolver
    sm = factory(device)
    sp = factory(device)
    sm.set_option(OPT_PRECISION, m_precision)
    if learned is not None:
        sp.gnn_set_params(learned)
    hist = []
    t_solve_m = t_solve_p = t_asm = 0.0
    t0 = time.time()
    for k in range(n_outer):
        ta = time.time()
        gradp = grad_p(p)
        M, rhs, Fm = momentum_field(m, u, flux=F, rho=rho, mu=mu, u_lid=u_lid, urf=urf_u)
        if F is None:
            F = Fm
        rhs -= gradp * vol[:, None]
        if reference_terms:
            rhs += momentum_deferred(m, u, gradient_sweeps(m, u, 2, 0, wall_u), F, mu)
        t_asm += time.time() - ta
        ts = time.time()
        if k == 0:
            sm.matrix_set(M)
        else:
            sm.matrix_values(M.p, M.n, M.pl)
        phi = np.ascontiguousarray(u)
        res0 = np.asfortranarray(rhs)
        rn_m = np.zeros(3)
        stm = sm.solv_bicg(2, m_reduc, m_iter, phi, res0, rn_m)
        u = phi
        t_solve_m += time.time() - ts
        ta = time.time()
        F = face_flux(m, u, p, gradp, M.pl, rho, aux=reference_terms)
        P = pressure_correction(m, M.pl, rho=rho, pin=1)
        b, imb = mass_imbalance(m, F, pin=1)
        t_asm += time.time() - ta
        ts = time.time()
        if k == 0:
            sp.matrix_set(P)
        else:
            sp.matrix_values(P.p, P.n, P.pl)
        pp = np.zeros((N, 1))
        sc = rhs_scale(N, imb) if p_scale else 1.0
        res0 = np.asfortranarray(b.reshape(-1, 1) * sc)
        rn_p = np.zeros(1)
        if learned is not None:
            stp = sp.solv_fcg(p_reduc, p_iter, pp, res0, rn_p, not_r0=True)
        else:
            stp = sp.solv_cg(p_imat, p_reduc, p_iter, pp, res0, rn_p, not_r0=True)
        pp /= sc
        t_solve_p += time.time() - ts
        ta = time.time()
        gradpp = grad_p(pp[:, 0])
        simple_correct(m, pp[:, 0].copy(), gradpp, M.pl, rho, urf_p, u, p, F)
        t_asm += time.time() - ta
        rec = {"it": k, "mass": float(imb), "mom_res0": rn_m.tolist(), "p_iters": stp["iters"][0],
               "m_iters": stm["iters"], "fallbacks": stp.get("fallbacks", 0)}
        hist.append(rec)
        if log_every and (k % log_every == 0 or k == n_outer - 1):
            print(json.dumps(rec), flush=True)
    sm.close()
    sp.close()
    timing = {"total_s": time.time() - t0, "assembly_s": t_asm, "momentum_solve_s": t_solve_m,
              "pressure_solve_s": t_solve_p, "n_cell": N}
    return u, p, hist, timing


def run_device(size=32, n_outer=200, re=1000.0, u_lid=1.0, urf_u=0.7, urf_p=0.3, jitter=0.15,
               seed=0, p_reduc=1e-10, p_iter=20000, m_reduc=0.1, m_iter=5, learned=None,
               p_imat=1, m_precision=0, device=0, log_every=0, reference_weights=False,
               reference_terms=False, renumber="rcm", p_scale=False, fcg_delta=None,
               p_options=None):
    """The same outer loop with everything on the GPU: assembly, gradients
    (the corrected sweeps too), the explicit momentum terms, fluxes and
    corrections by the fv_gpu kernels (bit-for-bit the host functions),
    solves through the device-pointer entry points; only the mass-imbalance
    norm comes back per iteration.  Same arguments and returns as run();
    renumber "color" takes the multicolour cell order (two-level DIC / DILU
    recurrences); timings are wall clock with the stream synchronised.
    p_options: further {option key: value} for the pressure solver."""
    import torch

    from .fv import GpuFv
    from .mesh import FaceMatrix
    rho = 1.0
    mu = rho * u_lid * 1.0 / re
    m = Mesh.hex(size, jitter=jitter, seed=seed, permute=True)
    m.renumber(Mesh.COLOR if renumber == "color" else Mesh.RCM)
    if reference_weights:
        m.set_face_weights(True)
    m.cache_geometry()
    N = m.n_cell
    ip, inb = m.faces()
    _, vol_h = m.cell_geom()
    wall_u = None
    if reference_terms:  # no-slip walls, the y = 1 lid moving (velocity wall values)
        _, nrm, xf, _, _ = m.face_geom()
        wall_h = np.zeros((m.n_face, 3))
        wall_h[(inb == 0) & (nrm[:, 1] > 0.9) & (xf[:, 1] > 1.0 - 1e-9), 0] = u_lid
    dev = torch.device("cuda", device)
    stream = torch.cuda.Stream(device=dev)
    fv = GpuFv(m, device)
    fv._lib.fv_gpu_set_stream(fv._h, stream.cuda_stream)
    sm = GpuSolver(device)
    sp = GpuSolver(device)
    for s_ in (sm, sp):
        s_.set_stream(stream.cuda_stream)
    sm.set_option(OPT_PRECISION, m_precision)
    if fcg_delta is not None:
        sp.set_option(OPT_FCG_RELIABLE_DELTA, fcg_delta)
    if learned is not None:
        sp.gnn_set_params(learned)
        # a stalled learned solve hands over to the plain run's own PCG
        sp.set_option(OPT_FCG_FALLBACK, max(0, min(int(p_imat), 2)))
    for key, value in (p_options or {}).items():  # further pressure-solver options
        sp.set_option(key, value)
    # the structure once (values come from the device each iteration)
    F_ = ip.shape[0]
    shell = FaceMatrix(N, ip, inb, np.zeros(F_), np.zeros(F_), np.ones(N))
    sm.matrix_set(shell)
    sp.matrix_set(shell)
    hist = []
    t_asm = t_solve_m = t_solve_p = 0.0

    def sync_time(t):
        stream.synchronize()
        return time.time() - t

    if reference_terms:
        grad_p = lambda q: fv.gradient_sweeps(q, 2, 2)
    else:
        grad_p = fv.gradient
    with torch.cuda.stream(stream):
        vol = torch.from_numpy(vol_h).to(dev)
        if reference_terms:
            wall_u = torch.from_numpy(wall_h).to(dev)
        u = torch.zeros(N, 3, dtype=torch.float64, device=dev)
        p = torch.zeros(N, dtype=torch.float64, device=dev)
        F = None
        t0 = time.time()
        for k in range(n_outer):
            ta = time.time()
            gradp = grad_p(p)
            Mp, Mn, Mpl, rhs, Fm = fv.momentum_field(u, flux=F, rho=rho, mu=mu, u_lid=u_lid,
                                                     urf=urf_u)
            if F is None:
                F = Fm
            rhs -= gradp * vol[:, None]
            if reference_terms:  # summed apart, then added, as the host loop does
                dcor = torch.zeros_like(rhs)
                fv.momentum_deferred(u, fv.gradient_sweeps(u, 2, 0, wall_u), F, mu, dcor)
                rhs += dcor
            t_asm += sync_time(ta)
            ts = time.time()
            sm.matrix_values_dev(Mp.data_ptr(), Mn.data_ptr(), Mpl.data_ptr())
            res0 = rhs.t().contiguous()  # column-major res0(ip, ivc)
            rn_m, stm = sm.solv_bicg_dev(2, m_reduc, m_iter, 3, u.data_ptr(), res0.data_ptr())
            t_solve_m += sync_time(ts)
            ta = time.time()
            F = fv.face_flux(u, p, gradp, Mpl, rho, aux=reference_terms)
            Pp, Pn, Ppl = fv.pressure_correction(Mpl, rho=rho, pin=1)
            b, imb = fv.mass_imbalance(F, pin=1)
            t_asm += sync_time(ta)
            ts = time.time()
            sp.matrix_values_dev(Pp.data_ptr(), Pn.data_ptr(), Ppl.data_ptr())
            pp = torch.zeros(N, dtype=torch.float64, device=dev)
            sc = rhs_scale(N, imb) if p_scale else 1.0
            if sc != 1.0:
                b *= sc
            if learned is not None:
                rn_p, stp = sp.solv_fcg_dev(p_reduc, p_iter, pp.data_ptr(), b.data_ptr(),
                                            not_r0=True)
            else:
                rn_p, stp = sp.solv_cg_dev(p_imat, p_reduc, p_iter, 1, pp.data_ptr(),
                                           b.data_ptr(), not_r0=True)
            if sc != 1.0:
                pp /= sc
            t_solve_p += sync_time(ts)
            ta = time.time()
            gradpp = grad_p(pp)
            fv.simple_correct(pp, gradpp, Mpl, rho, urf_p, u, p, F)
            t_asm += sync_time(ta)
            rec = {"it": k, "mass": float(imb), "mom_res0": list(map(float, rn_m)),
                   "p_iters": stp["iters"][0], "m_iters": stm["iters"],
                   "fallbacks": stp.get("fallbacks", 0),
                   "p_refinements": stp.get("refinements", 0)}
            hist.append(rec)
            if log_every and (k % log_every == 0 or k == n_outer - 1):
                print(json.dumps(rec), flush=True)
        total = sync_time(t0)
    u_h, p_h = u.cpu().numpy(), p.cpu().numpy()
    sm.close()
    sp.close()
    fv.close()
    timing = {"total_s": total, "assembly_s": t_asm, "momentum_solve_s": t_solve_m,
              "pressure_solve_s": t_solve_p, "n_cell": N}
    return u_h, p_h, hist, timing


def rhs_scale(n_cell, total):
    """The power of two nearest n_cell / total (1 for a zero total)."""
    if not total > 0:
        return 1.0
    return float(2.0 ** int(round(np.log2(n_cell / total))))


def rel_l2(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=32)
    ap.add_argument("--outer", type=int, default=200)
    ap.add_argument("--re", type=float, default=1000.0)
    ap.add_argument("--learned", action="store_true", help="also run learned + mixed FCG and compare")
    ap.add_argument("--weights", default=None)
    ap.add_argument("--log-every", type=int, default=20)
    ap.add_argument("--device-assembly", action="store_true",
                    help="assembly, gradients and corrections on the GPU too")
    ap.add_argument("--p-reduc", type=float, default=1e-10,
                    help="pressure solve tolerance (the reference's loop uses 0.1)")
    ap.add_argument("--p-iter", type=int, default=20000, help="(the reference: 20)")
    ap.add_argument("--p-imat", type=int, default=1, help="plain pressure PCG: 0 Jacobi, 1 DIC")
    ap.add_argument("--m-reduc", type=float, default=0.1)
    ap.add_argument("--m-iter", type=int, default=5)
    ap.add_argument("--reference-terms", action="store_true",
                    help="the reference's explicit momentum terms, corrected gradients and "
                         "auxiliary-point face pressures")
    ap.add_argument("--renumber", default="rcm", choices=["rcm", "color"],
                    help="cell order of the device loop's mesh")
    ap.add_argument("--p-scale", action="store_true",
                    help="normalise each pressure right-hand side by an exact power of two")
    ap.add_argument("--learned-m-precision", type=int, default=1,
                    help="momentum solves of the learned run: 1 FP32 inner iterations with "
                         "FP64 refinement, 0 FP64")
    ap.add_argument("--reference-weights", action="store_true",
                    help="the reference's face distance and interpolation weight")
    ap.add_argument("--fcg-delta", type=float, default=None,
                    help="device loop, learned run: the flexible CG's reliable-update drop "
                         "(SOLV_OPT_FCG_RELIABLE_DELTA; default the library's)")
    a = ap.parse_args(argv)
    loop = run_device if a.device_assembly else run
    kw = dict(p_reduc=a.p_reduc, p_iter=a.p_iter, p_imat=a.p_imat, m_reduc=a.m_reduc,
              m_iter=a.m_iter, log_every=a.log_every, reference_weights=a.reference_weights,
              p_scale=a.p_scale)
    if a.reference_terms:
        kw["reference_terms"] = True
    if a.device_assembly:
        kw["renumber"] = a.renumber
        if a.fcg_delta is not None:
            kw["fcg_delta"] = a.fcg_delta
    u0, p0, h0, t0 = loop(a.size, a.outer, a.re, **kw)
    out = {"size": a.size, "outer": a.outer, "re": a.re, "p_reduc": a.p_reduc,
           "p_imat": a.p_imat, "reference_terms": a.reference_terms, "p_scale": a.p_scale,
           "renumber": a.renumber if a.device_assembly else "rcm",
           "plain": t0, "final_mass_plain": h0[-1]["mass"], "first_mass": h0[0]["mass"],
           "p_iters_plain": int(np.sum([h["p_iters"] for h in h0]))}
    if a.learned:
        from .learn import DEFAULT_WEIGHTS, load_params
        w = load_params(a.weights or DEFAULT_WEIGHTS)
        u1, p1, h1, t1 = loop(a.size, a.outer, a.re, learned=w,
                              m_precision=a.learned_m_precision, **kw)
        out.update(learned=t1, p_iters_learned=int(np.sum([h["p_iters"] for h in h1])),
                   fallbacks=int(np.sum([h["fallbacks"] for h in h1])),
                   m_precision_learned=a.learned_m_precision,
                   final_mass_learned=h1[-1]["mass"],
                   rel_l2_u=rel_l2(u1[:, 0], u0[:, 0]), rel_l2_v=rel_l2(u1[:, 1], u0[:, 1]),
                   rel_l2_w=rel_l2(u1[:, 2], u0[:, 2]), rel_l2_p=rel_l2(p1, p0))
    print(json.dumps(out))


if __name__ == "__main__":
    main()
