"""Generates the golden fixtures in tests/golden/ from the REFERENCE's own code.

Runs the binaries that `make -C oracle ref` builds in oracle/_ref/ from the
reference sources (only its absent meshProcessor submodule is replaced by
oracle/ref_stub/):
  * ref_dump            AngularData, LebedevQuad, HemiQuad, Spherical, xE1,
                        trieig, Config, MeshData + ComputeMoments/ComputeFlux;
  * fp64/transfer_ref_cpu
                        the reference program (main.cpp: CG / invprec /
                        moments / flux), its kernels executed by the oracle.
Usage:  python tests/golden/make_golden.py      (needs the reference tree)
"""
import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def run(*args, cwd=None):
    p = subprocess.run(list(args), cwd=cwd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(f"{args} failed ({p.returncode}):\n{p.stdout[-2000:]}\n{p.stderr[-2000:]}")
    return p.stdout


def read_bin(path):
    return open(path, "rb").read()


def dump_angular(tmp):
    for k in range(0, 8):
        fn = os.path.join(tmp, f"ang{k}.bin")
        run(os.path.join(REF, "ref_dump"), "angular", str(k), fn)
        b = read_bin(fn)
        n = int(np.frombuffer(b[:4], np.int32)[0])
        o = 4
        om = np.frombuffer(b[o:o + 24 * n * n], np.float64).reshape(3, n, n); o += 24 * n * n
        pos = np.frombuffer(b[o:o + 12 * n * n], np.uint32).reshape(3, n, n); o += 12 * n * n
        O = np.frombuffer(b[o:o + 24 * n * n], np.float64).reshape(3, n, n)
        np.savez_compressed(os.path.join(HERE, f"angular_maxk{k}.npz"), slm=n, omega=om, omega_pos=pos,
                            Ox=O[0], Oy=O[1], Oz=O[2])


def dump_rules(tmp):
    out = {}
    for mode, degs in (("lebedev", [2, 6, 10, 13, 14, 17, 18, 22, 25, 26, 29, 30]), ("hemi", [1, 5, 9, 13, 17, 21, 25, 29])):
        for d in degs:
            fn = os.path.join(tmp, f"{mode}{d}.bin")
            run(os.path.join(REF, "ref_dump"), mode, str(d), fn)
            b = read_bin(fn)
            n = int(np.frombuffer(b[:4], np.int32)[0])
            a = np.frombuffer(b[4:4 + 32 * n], np.float64).reshape(4, n)
            out[f"{mode}_{d}"] = a
    np.savez_compressed(os.path.join(HERE, "quadrature.npz"), **out)


def dump_misc(tmp):
    fn = os.path.join(tmp, "sph.bin")
    run(os.path.join(REF, "ref_dump"), "sph", "14", fn)
    b = read_bin(fn)
    L, npt = np.frombuffer(b[:8], np.int32)
    o = 8
    xyz = np.frombuffer(b[o:o + 24 * npt], np.float64).reshape(3, npt); o += 24 * npt
    vals = np.frombuffer(b[o:], np.float64).reshape((L + 1) ** 2, npt)
    fn = os.path.join(tmp, "xe1.bin")
    run(os.path.join(REF, "ref_dump"), "xe1", fn)
    b = read_bin(fn)
    n = int(np.frombuffer(b[:4], np.int32)[0])
    xs = np.frombuffer(b[4:4 + 8 * n], np.float64)
    xe1 = np.frombuffer(b[4 + 8 * n:4 + 16 * n], np.float64)
    fn = os.path.join(tmp, "tri.bin")
    run(os.path.join(REF, "ref_dump"), "trieig", fn)
    b = read_bin(fn)
    nc = int(np.frombuffer(b[:4], np.int32)[0])
    o, cases = 4, []
    for _ in range(nc):
        N = int(np.frombuffer(b[o:o + 4], np.int32)[0]); o += 4
        a = np.frombuffer(b[o:o + 8 * N], np.float64); o += 8 * N
        bb = np.frombuffer(b[o:o + 8 * N], np.float64); o += 8 * N
        lm = float(np.frombuffer(b[o:o + 8], np.float64)[0]); o += 8
        cases.append((a, bb, lm))
    np.savez_compressed(os.path.join(HERE, "misc.npz"), sph_L=L, sph_xyz=xyz, sph_vals=vals, xe1_x=xs, xe1=xe1,
                        trieig_a=np.concatenate([c[0] for c in cases]),
                        trieig_b=np.concatenate([c[1] for c in cases]),
                        trieig_n=np.array([len(c[0]) for c in cases]), trieig_l=np.array([c[2] for c in cases]))


CONFIGS = {
    "full": """# all keys
numregs = 3
meshfile = some mesh.vol
outfile = out put.vtk
device = 2
angorder = 4
soltype = 2
dump = 1
precondition = 1
tolerance = 1e-9
[region 1]
kappa = 11.5
Ip = 1
albedo = 0.5
[region 2]
kappa = 0.25
Ip = 0
[region 3]
Ip = 2.5e-3
kappa = 1e2
""",
    "minimal": "numregs = 1\nangorder = 2\nmeshfile = m.vol\n[region 1]\nkappa = 1\nIp = 3\n",
    "err_section_first": "[region 1]\nnumregs = 1\n",
    "err_region_range": "numregs = 1\n[region 2]\n",
    "err_kappa_outside": "numregs = 1\nkappa = 1\n",
    "err_bad_number": "numregs = 1\n[region 1]\nkappa = abc\n",
    "err_meshfile_in_section": "numregs = 1\n[region 1]\nmeshfile = x\n",
}


def dump_configs(tmp):
    res = {}
    for name, text in CONFIGS.items():
        if text is None:
            continue
        fn = os.path.join(HERE, f"cfg_{name}.cfg")
        with open(fn, "w") as f:
            f.write(text)
        p = subprocess.run([os.path.join(REF, "ref_dump"), "config", fn, "3"], capture_output=True, text=True)
        lines = [ln[7:] for ln in p.stdout.splitlines() if ln.startswith("RESULT ")]
        res[name] = {"returncode": p.returncode, "result": lines}
    with open(os.path.join(HERE, "configs.json"), "w") as f:
        json.dump(res, f, indent=1, sort_keys=True)


# input writers and output parsers of the reference program (shared with
# the GPU tests and the bench's reference measurements)
from ref_program import parse_fields, parse_log, ref_cfg, write_tmesh  # noqa: E402


CASES = {
    # name: (n, jitter, maxk, kappa, Ip, precondition, seed)
    "small_k1": ((4, 4, 4), 0.2, 1, [0.0, 1.0, 3.0], [0.0, 1.0, 0.0], 0, 7),
    "small_k2": ((3, 4, 5), 0.2, 2, [0.0, 2.0, 0.5], [0.0, 1.0, 0.25], 0, 11),
    "small_k1_prec": ((3, 3, 3), 0.15, 1, [0.0, 1.0, 2.0], [0.0, 1.0, 0.0], 1, 5),
    "c1_k1": ((16, 16, 16), 0.2, 1, [0.0, 1.0, 1.0], [0.0, 1.0, 0.0], 0, 20261203),
}


def case_mesh(name):
    import transfer_b200 as tr
    n, jit, maxk, kappa, Ip, prec, seed = CASES[name]
    box = (0, 1, 0, 1, 0, 1)
    return tr.MeshData.kuhn(n, box=box, jitter=jit, seed=seed, kappa=kappa, Ip=Ip, region_kind=1,
                            region_arg=(0.5, 0.5, 0.5, 0.3 if name != "c1_k1" else 0.25))


def dump_runs(tmp):
    for name, (n, jit, maxk, kappa, Ip, prec, seed) in CASES.items():
        md = case_mesh(name)
        mesh = os.path.join(tmp, f"{name}.tmesh")
        write_tmesh(md, mesh)
        cfg = ref_cfg(tmp, mesh, maxk, kappa, Ip, prec=prec)
        # MeshData built by the reference's MeshData.cpp + moments/flux
        if name.startswith("small"):
            out = os.path.join(tmp, f"{name}.md")
            run(os.path.join(REF, "ref_dump"), "meshdata", cfg, out)
            b = read_bin(out)
            o = 0

            def take(dtype, count):
                nonlocal o
                a = np.frombuffer(b[o:o + np.dtype(dtype).itemsize * count], dtype)
                o += np.dtype(dtype).itemsize * count
                return a
            nP, nT, nF = take(np.uint32, 3)
            tetstart = take(np.uint32, nP + 1)
            tetidx = take(np.uint32, int(tetstart[-1]))
            tetpos = take(np.uint32, int(tetstart[-1]))
            mesh_rec = take(np.uint8, 128 * nT)
            facestart = take(np.uint32, nP + 1)
            faceidx = take(np.uint32, int(facestart[-1]))
            facepos = take(np.uint32, int(facestart[-1]))
            bnd = take(np.uint8, 64 * nF)
            slm = int(take(np.uint32, 1)[0])
            I = take(np.float64, slm * nP).reshape(slm, nP)
            U = take(np.float64, nP)
            T = take(np.float64, 9 * nP).reshape(3, 3, nP)
            W = take(np.float64, 3 * nT).reshape(3, nT)
            np.savez_compressed(os.path.join(HERE, f"meshdata_{name}.npz"), coords=md.coords, tets=md.mesh["p"],
                                regions=md.regions, tetstart=tetstart, tetidx=tetidx, tetpos=tetpos,
                                mesh=mesh_rec, facestart=facestart, faceidx=faceidx, facepos=facepos, bnd=bnd,
                                I=I, U=U, T=T, W=W)
        # the reference program end to end (its CG stop: ||r|| < 1e-4)
        outf = os.path.join(tmp, f"{name}.sol")
        cfg = ref_cfg(tmp, mesh, maxk, kappa, Ip, prec=prec, out=outf)
        log = run(os.path.join(REF, "fp64", "transfer_ref_cpu"), cfg, cwd=tmp)
        ks, res, preck = parse_log(log)
        fl = parse_fields(outf)
        np.savez_compressed(os.path.join(HERE, f"refrun_{name}.npz"), k=ks, residual=res, preck=preck,
                            U=fl["U"], T=fl["T"], W=fl["W"], maxk=maxk, kappa=kappa, Ip=Ip, n=n, jitter=jit,
                            seed=seed, precondition=prec)


def main():
    if not os.path.exists(os.path.join(REF, "ref_dump")):
        sys.exit("oracle/_ref is not built: run `make -C oracle ref`")
    with tempfile.TemporaryDirectory() as tmp:
        dump_angular(tmp)
        dump_rules(tmp)
        dump_misc(tmp)
        dump_configs(tmp)
        dump_runs(tmp)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
