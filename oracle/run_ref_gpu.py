"""MEASUREMENT INFRASTRUCTURE, not product code: runs the reference's own
CUDA program on a workload mesh so that its kernels can be timed on the same
GPU as this library's (for example under ncu's launch list).

The program is oracle/_ref/<precision>/transfer_ref_gpu (the reference's
main.cpp, host code and driver-API CudaContext, built from its sources by
`make -C oracle ref`) with kernels.sm_100.cubin (the reference's kernels.cu
compiled for sm_100a).  It reads the mesh through oracle/ref_stub (the
reference's meshProcessor submodule is absent) and runs its CG loop
(main.cpp:125-160) to its absolute stop 1e-4.  The reference has no
inflow boundary condition, so the source is Ip = 1 in every cell.

  python oracle/run_ref_gpu.py [--workload milne_slab] [--precision fp64]
"""
import argparse
import importlib.util
import os
import shutil
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _make_golden():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(ROOT, "tests", "golden",
                                                                              "make_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def mesh_of(workload):
    import transfer_b200 as tr
    if workload == "milne_slab":
        md = tr.MeshData.kuhn((8, 8, 160), box=(0.0, 1.0, 0.0, 1.0, 0.0, 20.0), jitter=0.15, seed=20261203,
                              kappa=[0.0, 1.0], Ip=[0.0, 1.0])
        return md, 3, [0.0, 1.0], [0.0, 1.0]
    if workload == "config1":
        md = tr.MeshData.kuhn((16, 16, 16), jitter=0.2, seed=20261203, kappa=[0.0, 1.0, 1.0], Ip=[0.0, 1.0, 0.0],
                              region_kind=1, region_arg=(0.5, 0.5, 0.5, 0.25))
        return md, 1, [0.0, 1.0, 1.0], [0.0, 1.0, 0.0]
    raise SystemExit(f"unknown workload {workload}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="milne_slab")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    a = ap.parse_args()
    ref = os.path.join(ROOT, "oracle", "_ref", a.precision)
    exe, cubin = os.path.join(ref, "transfer_ref_gpu"), os.path.join(ref, "kernels.sm_100.cubin")
    if not (os.path.exists(exe) and os.path.exists(cubin)):
        raise SystemExit(f"{exe} is not built (make -C oracle ref)")
    mg = _make_golden()
    md, maxk, kappa, Ip = mesh_of(a.workload)
    with tempfile.TemporaryDirectory() as tmp:
        shutil.copy(cubin, os.path.join(tmp, "kernels.sm_100.cubin"))
        mesh = os.path.join(tmp, "m.tmesh")
        mg.write_tmesh(md, mesh)
        cfg = mg.ref_cfg(tmp, mesh, maxk, kappa, Ip, out=os.path.join(tmp, "sol.txt"))
        t0 = time.perf_counter()
        p = subprocess.run([exe, cfg], cwd=tmp, capture_output=True, text=True, timeout=600)
        wall = time.perf_counter() - t0
    if p.returncode != 0 or "failed with error" in p.stderr:
        sys.stderr.write(p.stdout[-2000:] + p.stderr[-2000:])
        raise SystemExit(1)
    ks, res, _ = mg.parse_log(p.stdout)
    print(f"{a.workload} {a.precision}: nP={md.nP} nT={md.nT} maxk={maxk}: {len(ks)} CG iterations, "
          f"final |r| {res[-1]:.3e}, program wall time {wall:.2f} s")


if __name__ == "__main__":
    main()
