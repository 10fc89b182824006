"""CPU checks of the benchmark's workload definitions and work models
(transfer_b200/workloads.py) and of bench.py's module-level helpers."""
import importlib.util
import os

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
    assert md.nT == 6 * 2 * 2 * 8 and len(ords[3]) == 112 and abs(ords[3].sum() - 1) < 1e-14
    assert (ph.face_bc == tr.TR_BC_REFLECTIVE).sum() == 4 * 2 * 8 * 2
    assert desc["workload"] == "milne_sweep"


def test_bench_module_imports():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    assert callable(bench.sweep_section) and callable(bench.run_ours) and callable(bench.run_reference)
