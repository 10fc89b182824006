"""Command-line runner of the discrete-ordinates sweep on the Milne slab
(used to profile the sweep kernel)."""
def _main():
    """python -m transfer_b200.run_sweep [--precision 32|64] [--sweeps N]: N sweeps
    of the Milne slab (workloads.milne_sweep) with a scattering source, and
    the mean device time of one sweep."""
    import argparse

    import torch

    from . import workloads as W
    from .sweep import Sweep
    ap = argparse.ArgumentParser(description=_main.__doc__)
    ap.add_argument("--precision", type=int, default=32, choices=(32, 64))
    ap.add_argument("--sweeps", type=int, default=3)
    args = ap.parse_args()
    md, ph, ords, desc = W.milne_sweep()
    S = Sweep(0, md, ords, ph)
    J = torch.rand(4 * S.nT, dtype=torch.float64, device="cuda:0")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.sweeps):
        S.apply(J, None, precision=args.precision)
    e1.record()
    torch.cuda.synchronize()
    print(f"{desc['workload']}: nT {S.nT}, nq {S.nq}, {S.max_levels} levels; FP{args.precision} sweep "
          f"{e0.elapsed_time(e1) / args.sweeps:.3f} ms (host-timed, includes the API call)")


if __name__ == "__main__":
    _main()
