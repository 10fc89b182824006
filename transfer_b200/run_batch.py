"""Command-line runner of the batched sweep (configuration 4's problems):
one launch for all problems against one call per problem."""


def _main():
    """python -m transfer_b200.run_batch [--count 64] [--lo 2000] [--hi 400000]
    [--precision 32|64] [--reps 5] [--solve TOL]: one sweep of every problem
    of workloads.cube_batch with tr_sweep_apply_batch (one kernel launch for
    all problems' ordinates) against looping tr_sweep_apply over the
    problems; CUDA-event times, the mean of `reps` repetitions after one
    warm-up, and whether the two give identical scalar fluxes.  With --solve:
    source iteration of all problems to relative change TOL with
    tr_sweep_solve_batch (one CUDA-graph replay per iteration) against
    tr_sweep_solve (source iteration) problem after problem."""
    import argparse
    import time

    import torch

    from . import workloads as W
    from . import _lib as L
    from .sweep import Sweep, sweep_apply_batch, sweep_solve_batch

    ap = argparse.ArgumentParser(description=_main.__doc__)
    ap.add_argument("--count", type=int, default=64)
    ap.add_argument("--lo", type=int, default=2000)
    ap.add_argument("--hi", type=int, default=400000)
    ap.add_argument("--precision", type=int, default=32, choices=(32, 64))
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--solve", type=float, default=0.0)
    args = ap.parse_args()
    t0 = time.time()
    probs, desc = W.cube_batch(args.count, args.lo, args.hi)
    sweeps = [Sweep(0, md, ords, ph) for md, ph, ords in probs]
    nT = sum(S.nT for S in sweeps)
    upd = sum(S.nT * S.nq for S in sweeps)
    print(f"{desc['workload']}: {len(sweeps)} problems, {nT} tets in all ({min(S.nT for S in sweeps)}-"
          f"{max(S.nT for S in sweeps)}), {sum(S.nq for S in sweeps)} ordinate blocks, {upd / 1e6:.0f} M "
          f"cell-ordinate updates per sweep of all; set-up {time.time() - t0:.0f} s", flush=True)
    Js = [torch.rand(4 * S.nT, dtype=torch.float64, device="cuda:0") for S in sweeps]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def batched():
        return sweep_apply_batch(sweeps, args.precision, Js, None)

    def looped():
        return [S.apply(J, None, precision=args.precision) for S, J in zip(sweeps, Js)]
    res = {}
    for name, fn in (("batched", batched), ("looped", looped)):
        out = fn()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(args.reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.reps
        res[name] = (ms, out)
        print(f"{name}: {ms:.2f} ms per sweep of all problems, {upd / (ms * 1e-3) / 1e9:.2f} G updates/s", flush=True)
    same = all(torch.equal(a[0], b[0]) for a, b in zip(res["batched"][1], res["looped"][1]))
    print(f"speed-up of the single launch: {res['looped'][0] / res['batched'][0]:.2f}x; identical results: {same}")
    if args.solve > 0.0:
        mode = L.TR_MODE_FP64 if args.precision == 64 else L.TR_MODE_MIXED
        sweep_solve_batch(sweeps, args.precision, tol=args.solve, max_iter=2000)   # warm-up
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        e0.record()
        out, its, rr = sweep_solve_batch(sweeps, args.precision, tol=args.solve, max_iter=2000)
        e1.record()
        torch.cuda.synchronize()
        tb, wb = e0.elapsed_time(e1), (time.perf_counter() - t1) * 1e3
        t1 = time.perf_counter()
        e0.record()
        reps = [S.solve(method=L.TR_SWEEP_SOURCE_ITERATION, mode=mode, tol=args.solve, max_iter=2000) for S in sweeps]
        e1.record()
        torch.cuda.synchronize()
        tl, wl = e0.elapsed_time(e1), (time.perf_counter() - t1) * 1e3
        dev = max(float(((J - Jr).abs().max() / Jr.abs().max()).item()) for (J, _), (Jr, _, _) in zip(out, reps))
        print(f"source iteration to {args.solve:g}: batched {tb:.0f} ms ({int(its.max())} iterations, graph replays), "
              f"one problem after another {tl:.0f} ms ({sum(r[2].iterations for r in reps)} iterations in all); "
              f"{tl / tb:.2f}x; largest difference in J {dev:.1e}")


if __name__ == "__main__":
    _main()
