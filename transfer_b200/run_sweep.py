"""Command-line runner of the discrete-ordinates sweep on the Milne slab
(used to profile the sweep kernel and the accelerated solve)."""
def _main():
    """python -m transfer_b200.run_sweep [--precision 32|64] [--sweeps N]
    [--solve none|gmres|dsa] [--tol T]: N sweeps of the Milne slab
    (workloads.milne_sweep) with a scattering source and the mean device time
    of one sweep; with --solve, one GMRES solve to FP64 relative residual T in
    the given precision (64: FP64, 32: mixed), plain or with the diffusion
    synthetic acceleration."""
    import argparse

    import torch

    from . import _lib as L
    from . import workloads as W
    from .sweep import Sweep
    ap = argparse.ArgumentParser(description=_main.__doc__)
    ap.add_argument("--precision", type=int, default=32, choices=(32, 64))
    ap.add_argument("--sweeps", type=int, default=3)
    ap.add_argument("--solve", default="none", choices=("none", "gmres", "dsa"))
    ap.add_argument("--tol", type=float, default=1e-8)
    args = ap.parse_args()
    md, ph, ords, desc = W.milne_sweep()
    S = Sweep(0, md, ords, ph, dsa=args.solve == "dsa")
    J = torch.rand(4 * S.nT, dtype=torch.float64, device="cuda:0")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.sweeps):
        S.apply(J, None, precision=args.precision)
    e1.record()
    torch.cuda.synchronize()
    print(f"{desc['workload']}: nT {S.nT}, nq {S.nq}, {S.max_levels} levels; FP{args.precision} sweep "
          f"{e0.elapsed_time(e1) / max(args.sweeps, 1):.3f} ms (host-timed, includes the API call)")
    if args.solve != "none":
        mode = L.TR_MODE_FP64 if args.precision == 64 else L.TR_MODE_MIXED
        prec = L.TR_SWEEP_PREC_DSA if args.solve == "dsa" else L.TR_SWEEP_PREC_NONE
        _, _, rep = S.solve(mode=mode, tol=args.tol, restart=40, max_iter=5000, precondition=prec)
        print(f"solve ({args.solve}, FP{args.precision} sweeps): {rep.iterations} Krylov steps, "
              f"{rep.sweeps_f32} FP32 + {rep.sweeps_f64} FP64 sweeps, {rep.precond_solves} diffusion solves "
              f"({rep.precond_iterations} CG iterations), residual {rep.residual:.2e}, {rep.device_ms:.1f} ms")


if __name__ == "__main__":
    _main()
