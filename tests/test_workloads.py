"""CPU checks of the benchmark's workload definitions and work models
(transfer_b200/workloads.py) and of bench.py's module-level helpers."""
import importlib.util
import os

import numpy as np

import transfer_b200 as tr
from transfer_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_work_models_count_the_documented_bytes():
    md, ad, _, _ = W.config1(n=4)
    byt, flops = W.algorithmic_work(md, ad, real_bytes=8)
    assert byt == 16 * md.nP * ad.slm + 24 * md.nT + 24 * md.nP + 12 * md.nF and flops > 0
    ib, _ = W.cg_iteration_work(md, ad, real_bytes=4)
    assert ib == W.algorithmic_work(md, ad, real_bytes=4)[0] + 40 * md.nP * ad.slm
    sb, sf = W.sweep_work(61440, 112, real_bytes=4)
    assert sb == 112 * 61440 * 32 + 61440 * 80 and sf == 220 * 112 * 61440


def test_milne_sweep_workload():
    md, ph, ords, desc = W.milne_sweep(n=(2, 2, 8))
    assert md.nT == 6 * 2 * 2 * 8 and len(ords[3]) == 110 and abs(ords[3].sum() - 1) < 1e-14   # Lebedev 110
    # mirror-symmetric, as the reflective walls need
    pts = np.round(np.stack(ords[:3], axis=1), 12)
    assert {tuple(p) for p in pts} == {(-p[0], p[1], p[2]) for p in pts} == {(p[0], -p[1], p[2]) for p in pts}
    assert (ph.face_bc == tr.TR_BC_REFLECTIVE).sum() == 4 * 2 * 8 * 2
    assert desc["workload"] == "milne_sweep"


def test_bench_module_imports():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    assert callable(bench.sweep_section) and callable(bench.run_ours) and callable(bench.run_reference)


def test_sweep_workloads_at_small_sizes():
    """The stellar sphere and the cube64 sweep problem, built small: the ball
    keeps only tets inside r <= 1, coefficients follow the stated profiles,
    the functional covers the x = 1 faces, the 194-point set sums to 1."""
    from transfer_b200 import workloads as W
    md, ph, ords, desc = W.stellar_sphere(n=8, n_polar=2, n_azim=4)
    cent = md.coords[md.mesh["p"].astype(np.int64)].mean(axis=1)
    assert (np.linalg.norm(cent, axis=1) <= 1.0 + 1e-12).all() and len(ords[3]) == 8
    ratio = np.asarray(ph.kappa_abs_volume) / md.mesh["kappa_volume"]
    assert np.allclose(ratio, 2.0 / 3.0)
    md, ph, ords, mask, desc = W.cube64_sweep(n=6)
    assert len(ords[3]) == 194 and abs(ords[3].sum() - 1.0) < 1e-12
    fx = md.coords[md.bnd["p"][:, :3].astype(np.int64)][..., 0]
    assert mask.sum() == 2 * 6 * 6 and (fx[mask.astype(bool)] > 1 - 1e-9).all()


def test_runner_command_lines_parse():
    """The measurement runners start and print their usage without a GPU."""
    import subprocess
    import sys
    for mod in ("transfer_b200.run_sweep", "transfer_b200.run_batch", "transfer_b200.run_adjoint"):
        r = subprocess.run([sys.executable, "-m", mod, "--help"], cwd=os.path.dirname(os.path.dirname(__file__)),
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0 and "usage" in r.stdout, (mod, r.stderr[-500:])


def test_cube_batch_groups():
    """Configuration 4's problems carry 8 frequency groups: sigma_t scaled by
    10^(g/3 - 1) from one lognormal base, the problem's albedo in every group."""
    probs, desc = W.cube_batch(count=3, lo=50, hi=400, groups=8)
    assert desc["groups"] == 8 and len(probs) == 3
    for md, ph, ords, gc in probs:
        assert len(gc) == 7 and len(ords[3]) in (50, 194)
        kv0 = md.mesh["kappa_volume"]
        albedo = 1.0 - ph.kappa_abs_volume / kv0
        assert np.allclose(albedo, albedo[0]) and 0.0 <= albedo[0] <= 0.9
        for g, (kv, kav) in enumerate(gc, start=1):
            assert np.allclose(kv / kv0, 10.0 ** (g / 3.0))
            assert np.allclose(1.0 - kav / kv, albedo[0])
