"""Command-line runner of the discrete-ordinates sweep on the Milne slab or
the stellar sphere (used to profile the sweep kernel, the moments
contraction and the accelerated solve)."""
def _main():
    """python -m transfer_b200.run_sweep [--workload milne|stellar[:n]]
    [--precision 32|64] [--sweeps N] [--moments K] [--solve none|gmres|dsa]
    [--tol T] [--autotune] [--moments-kernel tcgen05|mma_sync]: N sweeps of the workload (workloads.milne_sweep, or
    workloads.stellar_sphere with n^3 grid cells, default 96) with a
    scattering source and the mean device time of one sweep; --moments: K
    launches of the l <= 3 moment contraction of the last sweep's psi, timed
    with CUDA events; with --solve, one GMRES solve to FP64 relative residual
    T in the given precision (64: FP64, 32: mixed), plain or with the
    diffusion synthetic acceleration; --autotune times both FP32 sweep shapes
    first and keeps the faster; --moments-kernel picks the tensor-core
    kernel family of the FP32 moments (tr_sweep_set_moments_kernel)."""
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
    ap.add_argument("--workload", default="milne")
    ap.add_argument("--moments", type=int, default=0)
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--moments-kernel", default="tcgen05", choices=("tcgen05", "mma_sync", "tma_ffma2"))
    args = ap.parse_args()
    if args.workload.startswith("stellar"):
        n = int(args.workload.split(":")[1]) if ":" in args.workload else 96
        md, ph, ords, desc = W.stellar_sphere(n=n)
    else:
        md, ph, ords, desc = W.milne_sweep()
    S = Sweep(0, md, ords, ph, dsa=args.solve == "dsa")
    S.set_moments_kernel({"tcgen05": L.TR_MOMENTS_TCGEN05, "mma_sync": L.TR_MOMENTS_MMA_SYNC,
                          "tma_ffma2": L.TR_MOMENTS_TMA_FFMA2}[args.moments_kernel])
    if args.autotune:
        shape, t_full, t_small = S.autotune()
        print(f"autotune: FP32 sweep {t_full:.3f} ms full shape, {t_small:.3f} ms small; keeps "
              f"{'small' if shape else 'full'}")
    J = torch.rand(4 * S.nT, dtype=torch.float64, device="cuda:0")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.sweeps):
        S.apply(J, None, precision=args.precision)
    e1.record()
    torch.cuda.synchronize()
    print(f"{desc['workload']}: nT {S.nT}, nq {S.nq}, {S.max_levels} levels; FP{args.precision} sweep "
          f"{e0.elapsed_time(e1) / max(args.sweeps, 1):.3f} ms (host-timed, includes the API call)")
    if args.moments:
        from ._lib import lib
        out = torch.zeros(16 * 4 * S.nT, dtype=torch.float64, device="cuda:0")
        S._c(lib.tr_sweep_moments(S._h, 16, out.data_ptr()))
        torch.cuda.synchronize()
        e0.record()
        for _ in range(args.moments):
            S._c(lib.tr_sweep_moments(S._h, 16, out.data_ptr()))
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.moments
        rb = 4 if args.precision == 32 else 8
        byt = S.nq * S.nT * 4 * rb + 16 * S.nT * 4 * 8
        print(f"moments l<=3 of FP{args.precision} psi ({args.moments_kernel if args.precision == 32 else 'fp64'}): "
              f"{ms:.3f} ms per launch (API call included), "
              f"{byt / (ms * 1e-3) / 1e9:.0f} GB/s algorithmic (psi read once, 16 FP64 moments written)")
    if args.solve != "none":
        mode = L.TR_MODE_FP64 if args.precision == 64 else L.TR_MODE_MIXED
        prec = L.TR_SWEEP_PREC_DSA if args.solve == "dsa" else L.TR_SWEEP_PREC_NONE
        _, _, rep = S.solve(mode=mode, tol=args.tol, restart=40, max_iter=5000, precondition=prec)
        print(f"solve ({args.solve}, FP{args.precision} sweeps): {rep.iterations} Krylov steps, "
              f"{rep.sweeps_f32} FP32 + {rep.sweeps_f64} FP64 sweeps, {rep.precond_solves} diffusion solves "
              f"({rep.precond_iterations} CG iterations), residual {rep.residual:.2e}, {rep.device_ms:.1f} ms")


if __name__ == "__main__":
    _main()
