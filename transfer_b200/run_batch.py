"""Command-line runner of the batched sweep (configuration 4's problems):
every (problem, frequency group) pair in one launch against one call per
pair."""


def build(count=64, lo=2000, hi=400000, groups=8):
    """Sweeps of workloads.cube_batch: per problem its sweep (group 0) and
    its groups 1 .. groups-1 (tr_sweep_create_group, sharing the problem's
    schedule).  Returns (sweeps, description)."""
    from . import workloads as W
    from .sweep import Sweep
    probs, desc = W.cube_batch(count, lo, hi, groups=groups)
    sweeps = []
    for md, ph, ords, gc in probs:
        S = Sweep(0, md, ords, ph)
        sweeps.append(S)
        sweeps += [S.create_group(kv, kav) for kv, kav in gc]
    return sweeps, desc


def _main():
    """python -m transfer_b200.run_batch [--count 64] [--lo 2000] [--hi 400000]
    [--groups 8] [--precision 32|64] [--reps 5] [--autotune] [--solve TOL]:
    one sweep of every (problem, group) of workloads.cube_batch with
    tr_sweep_apply_batch (one kernel launch for all their ordinates) against
    looping tr_sweep_apply over them; CUDA-event times, the mean of `reps`
    repetitions after one warm-up, and whether the two give identical scalar
    fluxes.  --autotune first times every launch form of the batch
    (tr_sweep_autotune_batch) and keeps the fastest.  With --solve: source
    iteration of all pairs to relative change TOL with tr_sweep_solve_batch
    (FP32 sweeps, FP64 iterates and stopping test; one CUDA-graph replay per
    iteration) against the plain FP64 solver (tr_sweep_solve, FP64 source
    iteration) looped over the pairs, each pair's work space released after
    its solve."""
    import argparse
    import time

    import torch

    from . import _lib as L
    from .sweep import sweep_apply_batch, sweep_autotune_batch, sweep_solve_batch

    ap = argparse.ArgumentParser(description=_main.__doc__)
    ap.add_argument("--count", type=int, default=64)
    ap.add_argument("--lo", type=int, default=2000)
    ap.add_argument("--hi", type=int, default=400000)
    ap.add_argument("--groups", type=int, default=8)
    ap.add_argument("--precision", type=int, default=32, choices=(32, 64))
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--solve", type=float, default=0.0)
    args = ap.parse_args()
    t0 = time.time()
    sweeps, desc = build(args.count, args.lo, args.hi, args.groups)
    nT = sum(S.nT for S in sweeps)
    upd = sum(S.nT * S.nq for S in sweeps)
    print(f"{desc['workload']}: {args.count} problems x {args.groups} groups = {len(sweeps)} sweeps, {nT} cell-groups "
          f"in all, {sum(S.nq for S in sweeps)} (problem, group, ordinate) tasks, {upd / 1e6:.0f} M cell-ordinate "
          f"updates per sweep of all; set-up {time.time() - t0:.0f} s", flush=True)
    if args.autotune:
        form, ms = sweep_autotune_batch(sweeps, args.precision)
        names = {0: "static/full", 1: "static/small", 2: "queue/full", 3: "queue/small"}
        print("autotune: " + ", ".join(f"{names[f]} {v:.2f} ms" for f, v in sorted(ms.items())) +
              f"; keeps {names[form]}", flush=True)
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
        print(f"{name}: {ms:.2f} ms per sweep of all pairs, {upd / (ms * 1e-3) / 1e9:.2f} G updates/s", flush=True)
    same = all(torch.equal(a[0], b[0]) for a, b in zip(res["batched"][1], res["looped"][1]))
    print(f"speed-up of the single launch: {res['looped'][0] / res['batched'][0]:.2f}x; identical results: {same}")
    if args.solve > 0.0:
        sweep_solve_batch(sweeps, 32, tol=args.solve, max_iter=2000)   # warm-up (and graph capture paths)
        torch.cuda.synchronize()
        e0.record()
        out, its, rr = sweep_solve_batch(sweeps, 32, tol=args.solve, max_iter=2000)
        e1.record()
        torch.cuda.synchronize()
        tb = e0.elapsed_time(e1)
        dev, tl, iters = 0.0, 0.0, 0
        for S, (J, _) in zip(sweeps, out):
            S.release_work()
            e0.record()
            Jr, _, rep = S.solve(method=L.TR_SWEEP_SOURCE_ITERATION, mode=L.TR_MODE_FP64, tol=args.solve,
                                 max_iter=2000)
            e1.record()
            torch.cuda.synchronize()
            tl += e0.elapsed_time(e1)
            iters += rep.iterations
            dev = max(dev, float(((J - Jr).abs().max() / Jr.abs().max()).item()))
            S.release_work()
        print(f"source iteration to {args.solve:g}: batched FP32 sweeps {tb:.0f} ms ({int(its.max())} iterations, "
              f"graph replays), FP64 solver pair after pair {tl:.0f} ms ({iters} iterations in all); "
              f"{tl / tb:.2f}x; largest difference in J {dev:.1e}")


if __name__ == "__main__":
    _main()
