"""Command-line runner of the adjoint gradient on the cube64 sweep problem
(workloads.cube64_sweep): timings and a central-difference check."""


def _main():
    """python -m transfer_b200.run_adjoint [--n 64] [--cells 32] [--step 1e-2]
    [--tol 1e-13]: forward and adjoint FP64 GMRES solves of the outflow through
    x = 1 on the n^3 cube (194-point Lebedev set), its gradient with respect
    to every cell's sigma_a and sigma_s in FP64 and FP32, then central
    differences F(sigma + h sigma) - F(sigma - h sigma) on `cells` seeded
    cells (drawn from the half x > 0.5, nearer the functional's faces) for
    both coefficients, each from its own FP64 solve after
    tr_sweep_set_coefficients."""
    import argparse
    import time

    import numpy as np
    import torch

    from . import _lib as L
    from . import workloads as W
    from .sweep import Sweep, adjoint_problem

    ap = argparse.ArgumentParser(description=_main.__doc__)
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--cells", type=int, default=32)
    ap.add_argument("--step", type=float, default=1e-2)
    ap.add_argument("--tol", type=float, default=1e-13)
    args = ap.parse_args()
    t0 = time.time()
    md, ph, ords, mask, desc = W.cube64_sweep(n=args.n)
    x, y, z, w = ords
    fwd = Sweep(0, md, ords, ph)
    md_adj, ph_adj = adjoint_problem(md, ph, mask)
    adj = Sweep(0, md_adj, (-x, -y, -z, w), ph_adj)
    print(f"{desc['workload']}: nT {fwd.nT}, nq {fwd.nq}, {fwd.max_levels} levels, {int(mask.sum())} functional "
          f"faces; set-up {time.time() - t0:.1f} s", flush=True)
    kw = dict(tol=args.tol, restart=30, max_iter=500)
    J, B, rf = fwd.solve(**kw)
    Ja, _, ra = adj.solve(**kw)
    _, _, rm = fwd.solve(mode=L.TR_MODE_MIXED, tol=1e-8, restart=30, max_iter=500)
    fwd.apply(J, B, precision=64)
    F = fwd.outflow(mask)
    print(f"forward FP64 solve: {rf.iterations} steps, {rf.device_ms:.0f} ms; adjoint: {ra.iterations} steps, "
          f"{ra.device_ms:.0f} ms; forward mixed to 1e-8: {rm.iterations} steps, {rm.device_ms:.0f} ms; "
          f"F = {F:.10e}", flush=True)
    grads = {}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for prec in (64, 32):
        ga, gs = fwd._dev(fwd.nT), fwd._dev(fwd.nT)
        e0.record()
        fwd._c(L.lib.tr_sweep_gradient(fwd._h, adj._h, prec, J.data_ptr(), B.data_ptr() if fwd.n_extra else None,
                                       Ja.data_ptr(), ga.data_ptr(), gs.data_ptr()))
        e1.record()
        torch.cuda.synchronize()
        grads[prec] = (ga[:fwd.nT].cpu().numpy(), gs[:fwd.nT].cpu().numpy())
        print(f"gradient FP{prec}: {e0.elapsed_time(e1):.1f} ms (two sweeps and the reduction)", flush=True)
    g64a, g64s = grads[64]
    g32a, g32s = grads[32]
    scale = max(np.abs(g64a).max(), np.abs(g64s).max())
    print(f"FP32 gradient vs FP64: max |diff| / max |grad| = "
          f"{max(np.abs(g32a - g64a).max(), np.abs(g32s - g64s).max()) / scale:.2e}", flush=True)
    # central differences on seeded cells
    tets = md.mesh["p"].astype(np.int64)
    cx = md.coords[tets].mean(axis=1)[:, 0]
    rng = np.random.default_rng(20261204)
    cells = rng.choice(np.flatnonzero(cx > 0.5), size=args.cells, replace=False)
    kv0 = md.mesh["kappa_volume"].astype(np.float64).copy()
    ka0 = np.asarray(ph.kappa_abs_volume, dtype=np.float64).copy()
    errs, worst = [], 0.0
    t1 = time.time()
    for c in cells:
        for which in ("sigma_a", "sigma_s"):
            part = ka0[c] if which == "sigma_a" else kv0[c] - ka0[c]   # sigma V of the perturbed coefficient
            Fs = []
            for sign in (1.0, -1.0):
                kv, ka = kv0.copy(), ka0.copy()
                d = sign * args.step * part
                kv[c] += d
                if which == "sigma_a":
                    ka[c] += d
                fwd.set_coefficients(kv, ka)
                Jp, Bp, rp = fwd.solve(**kw)
                fwd.apply(Jp, Bp, precision=64)
                Fs.append(fwd.outflow(mask))
            # the step in sigma V is d = step * part, in sigma d / V: dF/dsigma = V dF/d(sigma V)
            fd = (Fs[0] - Fs[1]) / (2.0 * args.step * part) * md_volume(md, c)
            adj_g = (g64a if which == "sigma_a" else g64s)[c]
            rel = abs(fd - adj_g) / max(abs(adj_g), 1e-300)
            errs.append(rel)
            worst = max(worst, rel)
    fwd.set_coefficients(kv0, ka0)
    errs = np.array(errs)
    print(f"central differences on {args.cells} cells x 2 coefficients (step {args.step:g} relative, FP64 solves "
          f"to {args.tol:g}, {time.time() - t1:.0f} s): relative error median {np.median(errs):.2e}, "
          f"max {worst:.2e}", flush=True)


def md_volume(md, c):
    """Volume of tet c from its vertex coordinates."""
    import numpy as np
    p = md.coords[md.mesh["p"][c].astype(np.int64)]
    return abs(np.linalg.det(np.stack([p[1] - p[0], p[2] - p[0], p[3] - p[0]]))) / 6.0


if __name__ == "__main__":
    _main()
