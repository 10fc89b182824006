"""Command-line runner of the even-parity operator alone (used to profile
k_lhs on one workload): python -m transfer_b200.run_operator
[--workload milne_slab_ref|milne_slab|config1|cube64] [--precision 64|32]
[--kind tensor|simt] [--reps 20].  Prints the mean CUDA-event time of one
application (tr_bench_lhs: back-to-back launches after 3 untimed ones) and
its algorithmic GB/s and TFLOP/s (workloads.algorithmic_work)."""


def _main():
    import argparse
    import ctypes as C

    import torch

    from . import _lib as L
    from . import workloads as W
    from .core import CudaContext

    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--workload", default="cube64", choices=sorted(W.WORKLOADS))
    ap.add_argument("--precision", type=int, default=64, choices=(32, 64))
    ap.add_argument("--kind", default="", choices=("", "tensor", "simt"))
    ap.add_argument("--reps", type=int, default=20)
    args = ap.parse_args()
    md, ad, phys, desc = W.WORKLOADS[args.workload]()
    ctx = CudaContext(0, md, ad, phys)
    if args.kind:
        L.check(L.lib.tr_ctx_set_operator(ctx._h, L.TR_OPERATOR_TENSOR if args.kind == "tensor"
                                          else L.TR_OPERATOR_SIMT), ctx._h)
    dt = torch.float64 if args.precision == 64 else torch.float32
    x = ctx.allocVector(dt)
    x.view(ctx.nP, -1)[:, :ctx.slm].normal_()
    y = ctx.allocVector(dt)
    ms = C.c_double()
    L.check(L.lib.tr_bench_lhs(ctx._h, args.precision, x.data_ptr(), y.data_ptr(), args.reps, C.byref(ms)), ctx._h)
    byt, flops = W.algorithmic_work(md, ad, real_bytes=args.precision // 8)
    t = ms.value * 1e-3
    print(f"{desc['workload']}: nP {ctx.nP}, nT {ctx.nT}, slm {ctx.slm}, edges {ctx.n_edges}; FP{args.precision} "
          f"operator {1e6 * t:.1f} us, {byt / t / 1e9:.0f} GB/s and {flops / t / 1e12:.2f} TFLOP/s algorithmic")
    ctx.close()


if __name__ == "__main__":
    _main()
