"""Runs the REFERENCE's own CUDA program on the GPU and checks both the
oracle and the product against it.

oracle/_ref/fp64/transfer_ref_gpu is the reference's main.cpp + host code +
CudaContext (CUDA driver API), built from the reference sources with only
its absent meshProcessor submodule replaced (oracle/ref_stub), and it loads
kernels.sm_100.cubin: the reference's kernels.cu compiled for sm_100a.
Built here by `make -C oracle ref`; the built files travel with the tree."""
import os
import shutil
import subprocess

import numpy as np
import pytest
import torch

import oracle_py as op
import ref_program as rp
import transfer_b200 as tr
from common import golden, golden_angular, refrun_mesh, rel_err

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")


def run_reference(tmp_path, precision, md, maxk, kappa, Ip, prec=0, dump=0):
    if rp.built(precision) is None:
        pytest.fail(f"oracle/_ref/{precision}/transfer_ref_gpu not built (make -C oracle ref)")
    r = rp.run_program(precision, md, maxk, kappa, Ip, prec=prec, dump=dump, workdir=tmp_path, timeout=300)
    assert r["returncode"] == 0, r["stdout"][-3000:] + r["stderr"][-3000:]
    assert "failed with error" not in r["stderr"], r["stderr"][-3000:]
    return r["k"], r["residual"], r["preck"], r["fields"], r


@pytest.mark.parametrize("name", ["small_k1", "small_k2", "small_k1_prec", "c1_k1"])
def test_reference_gpu_program_vs_oracle_and_product(cuda, tmp_path, name):
    r = golden(f"refrun_{name}.npz")
    md = refrun_mesh(r)
    maxk = int(r["maxk"])
    ks, res, preck, fl, _ = run_reference(tmp_path, "fp64", md, maxk, list(r["kappa"]), list(r["Ip"]),
                                          prec=int(r["precondition"]))
    # the reference's CUDA kernels vs the oracle's restatement of them (the
    # golden run is the same program with the oracle as its kernels)
    assert len(ks) == len(r["k"])
    assert abs(res[-1] / r["residual"][-1] - 1) < 1e-6
    loose = 1e-6 if name == "c1_k1" else 1e-7   # FMA contraction on the GPU, loose stop
    assert rel_err(fl["U"], r["U"]) < loose
    if int(r["precondition"]):
        assert preck == int(r["preck"])
    # the product with the reference's settings
    ctx = tr.CudaContext(0, md, golden_angular(maxk))
    f, rep = ctx.solve(tol=1e-4, precondition=int(r["precondition"]))
    assert rep.iterations == len(ks)
    U, _ = ctx.computeMoments(f)
    assert rel_err(U.cpu().numpy(), fl["U"]) < loose   # loose stop: see test_gpu_solver


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("fp32", 2e-6)])
def test_reference_gpu_operator_matrix(cuda, tmp_path, precision, tol):
    """The reference dumps its whole operator (dump = 1, main.cpp:73-104) by
    applying its kernels to unit vectors; compare every entry."""
    md = tr.MeshData.kuhn((2, 2, 3), jitter=0.2, seed=3, kappa=[0.0, 1.5, 0.7], Ip=[0.0, 1.0, 0.0],
                          region_kind=1, region_arg=(0.5, 0.5, 0.5, 0.4))
    maxk = 1
    run_reference(tmp_path, precision, md, maxk, [0.0, 1.5, 0.7], [0.0, 1.0, 0.0], dump=1)
    rows = np.loadtxt(tmp_path / "slae.dat")
    ad = golden_angular(maxk)
    slm = ad.slm
    aslm_ref = 8 if precision == "fp64" else 16
    cols = [k for k in range(md.nP * aslm_ref) if k % aslm_ref < slm]
    assert rows.shape == (len(cols), md.nP * slm + 1)
    ctx = tr.CudaContext(0, md, ad)
    ours = np.zeros((len(cols), md.nP * slm))
    for c, k in enumerate(cols):
        e = np.zeros((md.nP, ctx.aslm))
        e[k // aslm_ref, k % aslm_ref] = 1.0
        Af = ctx.allocVector()
        ctx.computeLhs(torch.from_numpy(e.reshape(-1)).cuda(), Af)
        ours[c] = Af.cpu().numpy().reshape(md.nP, ctx.aslm)[:, :slm].reshape(-1)
    assert rel_err(ours, rows[:, :-1]) < tol
    # and its right-hand side column
    b = ctx.allocVector()
    ctx.computeRhs(b)
    bb = b.cpu().numpy().reshape(md.nP, ctx.aslm)[:, :slm].reshape(-1)
    assert rel_err(bb, rows[:, -1]) < tol
