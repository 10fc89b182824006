"""TEST AND MEASUREMENT INFRASTRUCTURE, not product code: drives the
reference's own programs, built from its sources by `make -C oracle ref`
into oracle/_ref/ (only its absent meshProcessor submodule is replaced by
oracle/ref_stub/):

  <precision>/transfer_ref_gpu   the reference program (main.cpp + host code +
                                 driver-API CudaContext) with
  <precision>/kernels.sm_100.cubin
                                 the reference's kernels.cu for sm_100a;
  <precision>/ref_bench          its computeLhs and dot timed with CUDA
                                 events through its own CudaContext
                                 (oracle/ref_bench.cpp);
  fp64/transfer_ref_cpu          the reference program with the oracle as its
                                 kernels (CPU).

Input files: a plain-text mesh for the stand-in meshProcessor (write_tmesh)
and a radiation.cfg in the reference's grammar (ref_cfg).  Output parsing
follows the program's printf lines (main.cpp:125-160: "k = <k> norm r = <r>",
"preck = <n>") and the stand-in saveVtk text file (parse_fields).
"""
import os
import re
import shutil
import subprocess
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, "_ref")


def write_tmesh(md, path):
    """The stand-in meshProcessor's input (oracle/ref_stub/mesh.cpp)."""
    with open(path, "w") as f:
        f.write(f"tmesh 1\n{md.nP}\n")
        for x in md.coords:
            f.write(f"{x[0]:.17g} {x[1]:.17g} {x[2]:.17g}\n")
        f.write(f"{md.nT}\n")
        for t in range(md.nT):
            p = md.mesh["p"][t]
            f.write(f"{p[0]} {p[1]} {p[2]} {p[3]} {md.regions[t]}\n")


def ref_cfg(tmp, meshfile, maxk, kappa, Ip, prec=0, dump=0, out="sol.txt"):
    """A radiation.cfg for the reference (per-region kappa / Ip, index 0 unused)."""
    lines = [f"numregs = {len(kappa) - 1}", f"meshfile = {meshfile}", f"outfile = {out}", "device = 0",
             f"angorder = {maxk}", f"dump = {dump}", f"precondition = {prec}", "soltype = 0"]
    for r in range(1, len(kappa)):
        lines += [f"[region {r}]", f"kappa = {float(kappa[r])!r}", f"Ip = {float(Ip[r])!r}"]
    fn = os.path.join(tmp, "run.cfg")
    with open(fn, "w") as f:
        f.write("\n".join(lines) + "\n")
    return fn


def parse_fields(path):
    fields, cur, rows = {}, None, []
    for ln in open(path):
        parts = ln.split()
        if len(parts) == 4 and parts[0] in ("cell", "point"):
            if cur:
                fields[cur] = np.array(rows)
            cur, rows = parts[1], []
        else:
            rows.append(float(ln))
    if cur:
        fields[cur] = np.array(rows)
    return fields


def parse_log(text):
    ks = [(int(m.group(1)), float(m.group(2))) for m in re.finditer(r"^k = (\d+) norm r = (\S+)", text, re.M)]
    pre = re.search(r"^preck = (\d+)", text, re.M)
    return np.array([k for k, _ in ks]), np.array([r for _, r in ks]), int(pre.group(1)) if pre else -1


def built(precision, name="transfer_ref_gpu"):
    exe = os.path.join(REF, precision, name)
    cubin = os.path.join(REF, precision, "kernels.sm_100.cubin")
    return exe if os.path.exists(exe) and os.path.exists(cubin) else None


def _stage(tmp, precision, md, maxk, kappa, Ip, prec=0, dump=0):
    shutil.copy(os.path.join(REF, precision, "kernels.sm_100.cubin"), os.path.join(tmp, "kernels.sm_100.cubin"))
    mesh = os.path.join(tmp, "m.tmesh")
    write_tmesh(md, mesh)
    out = os.path.join(tmp, "sol.txt")
    return ref_cfg(tmp, mesh, maxk, kappa, Ip, prec=prec, dump=dump, out=out), out


def run_program(precision, md, maxk, kappa, Ip, prec=0, dump=0, workdir=None, timeout=600):
    """Runs the reference program on the GPU.  Its stdout is line-buffered
    (stdbuf) and each CG line is time-stamped as it arrives, so the CG loop's
    own wall time is measured apart from the program's set-up and output.
    Returns dict(k, residual, preck, fields, wall_s, cg_s, ms_per_iteration,
    stdout, stderr, returncode); ms_per_iteration covers the iterations
    between the first and the last CG line (each includes the reference's
    two blocking dot/norm read-backs)."""
    exe = built(precision)
    if exe is None:
        raise FileNotFoundError(f"oracle/_ref/{precision}/transfer_ref_gpu is not built (make -C oracle ref)")
    own = workdir is None
    tmp = tempfile.mkdtemp() if own else str(workdir)
    try:
        cfg, out = _stage(tmp, precision, md, maxk, kappa, Ip, prec=prec, dump=dump)
        cmd = [exe, cfg]
        if shutil.which("stdbuf"):
            cmd = ["stdbuf", "-oL"] + cmd
        t0 = time.perf_counter()
        p = subprocess.Popen(cmd, cwd=tmp, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
        lines, stamps = [], []
        deadline = t0 + timeout
        for ln in p.stdout:
            lines.append(ln)
            if ln.startswith("k = "):
                stamps.append(time.perf_counter())
            if time.perf_counter() > deadline:
                p.kill()
                break
        err = p.stderr.read()
        rc = p.wait()
        wall = time.perf_counter() - t0
        text = "".join(lines)
        ks, res, preck = parse_log(text)
        fields = parse_fields(out) if rc == 0 and os.path.exists(out) else {}
        per_it = 1e3 * (stamps[-1] - stamps[0]) / (len(stamps) - 1) if len(stamps) > 1 else None
        return dict(k=ks, residual=res, preck=preck, fields=fields, wall_s=wall,
                    cg_s=(stamps[-1] - stamps[0]) if len(stamps) > 1 else None, ms_per_iteration=per_it,
                    stdout=text, stderr=err, returncode=rc)
    finally:
        if own:
            shutil.rmtree(tmp, ignore_errors=True)


def bench_kernels(precision, md, maxk, kappa, Ip, reps=50, timeout=600):
    """The reference's computeLhs and dot timed through its own CudaContext
    (ref_bench): returns dict(lhs_ms, dot_ms, nP, aslm)."""
    exe = built(precision, "ref_bench")
    if exe is None:
        raise FileNotFoundError(f"oracle/_ref/{precision}/ref_bench is not built (make -C oracle ref)")
    tmp = tempfile.mkdtemp()
    try:
        cfg, _ = _stage(tmp, precision, md, maxk, kappa, Ip)
        p = subprocess.run([exe, cfg, str(reps)], cwd=tmp, capture_output=True, text=True, timeout=timeout)
        if p.returncode != 0 or "failed with error" in p.stderr:
            raise RuntimeError(f"ref_bench failed ({p.returncode}): {p.stdout[-1000:]} {p.stderr[-1000:]}")
        m = re.search(r"lhs_ms=(\S+) dot_ms=(\S+) nP=(\d+) aslm=(\d+)", p.stdout)
        return dict(lhs_ms=float(m.group(1)), dot_ms=float(m.group(2)), nP=int(m.group(3)), aslm=int(m.group(4)))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
