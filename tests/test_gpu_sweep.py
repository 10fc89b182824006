"""GPU parity of the discrete-ordinates sweep (transfer_b200/csrc/sweep.cu)
against the FP64 oracle (oracle/sweep_oracle.c), through the C ABI.

Tolerances: the device schedule is exact (same dependency levels, same lag
slots); one FP64 sweep agrees with the oracle to 1e-12 relative (FMA
contraction and the order of the face sums differ); one FP32 sweep to 2e-5;
converged FP64 solves to 1e-9; mixed (FP32 sweeps in FP64 defect
correction) solves reach an FP64 residual of 1e-8 with J within 1e-6 of the
oracle; the FP64 energy balance closes to 1e-12 of the emission."""
import numpy as np
import pytest
import torch

import oracle_py as op
import transfer_b200 as tr
from common import rel_err
from sweep_cases import absorbing_slab, diffusive_box, e2_slab_exact, scattering_box, tangled_cube, vertex_x

pytestmark = pytest.mark.gpu


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).cuda()


def host(t):
    return t.detach().cpu().numpy()


def pair(case, ords):
    md, ph = case
    S = tr.Sweep(0, md, ords, ph)
    O = op.SweepOracle(md, ords, kappa_abs_volume=ph.kappa_abs_volume, face_bc=ph.face_bc,
                       face_incident=ph.face_incident)
    return md, ph, S, O


@pytest.mark.parametrize("which", ["scattering_box", "absorbing_slab", "tangled_cube"])
def test_schedule_matches_oracle(cuda, which):
    case = {"scattering_box": scattering_box, "absorbing_slab": lambda: absorbing_slab(nx=12, ny=3, nz=2),
            "tangled_cube": tangled_cube}[which]()
    md, ph, S, O = pair(case, op.ordinates_product(4, 8))
    assert (S.n_extra, S.n_reflective, S.n_lag, S.max_levels, S.forced_levels) == \
        (O.nB, O.n_reflective, O.n_lag, O.max_levels, O.forced)
    assert np.array_equal(S.levels(), O.levels())


@pytest.mark.parametrize("which", ["scattering_box", "tangled_cube"])
def test_single_sweep_fp64_matches_oracle(cuda, which):
    case = scattering_box() if which == "scattering_box" else tangled_cube()
    md, ph, S, O = pair(case, op.ordinates_product(4, 8))
    rng = np.random.default_rng(3)
    Jin, Bin = rng.random((md.nT, 4)), rng.random(max(S.n_extra, 1))[:S.n_extra]
    for J0, B0, ext in ((None, None, 1), (Jin, Bin, 1), (Jin, Bin, 0)):
        Jg, Bg = S.apply(None if J0 is None else dev(J0), None if B0 is None else dev(B0), with_ext=ext)
        Jo, Bo, psio = O.apply(J0, B0, with_ext=ext, want_psi=True)
        assert rel_err(host(Jg), Jo) < 1e-12
        if S.n_extra:
            assert rel_err(host(Bg), Bo) < 1e-12
        assert rel_err(host(S.psi()), psio) < 1e-12


@pytest.mark.parametrize("n,polar,azim", [((5, 4, 6), 4, 8), ((5, 4, 6), 10, 16), ((8, 8, 8), 10, 16)])
def test_single_sweep_fp32_matches_oracle(cuda, n, polar, azim):
    """32 ordinates: one block per SM; 160 (more than the SMs): the small
    shared-memory shape with two blocks per SM and a ring of 1,024 positions,
    so on the 8^3 box (3,072 cells) upwind traces also come from global psi.
    (On the tangled cube FP32 differs from the oracle by up to 1e-4 with any
    shape: its inverted elements make some 4x4 systems ill-conditioned.)"""
    md, ph, S, O = pair(scattering_box(n=n), op.ordinates_product(polar, azim))
    rng = np.random.default_rng(4)
    Jin, Bin = rng.random((md.nT, 4)), rng.random(S.n_extra)
    Jg, Bg = S.apply(dev(Jin), dev(Bin), precision=32)
    Jo, Bo = O.apply(Jin, Bin)
    assert rel_err(host(Jg), Jo) < 2e-5
    assert rel_err(host(Bg), Bo) < 2e-5


def test_balance_matches_oracle_and_closes(cuda):
    md, ph, S, O = pair(scattering_box(), op.ordinates_product(4, 8))
    rng = np.random.default_rng(5)
    Jin, Bin = rng.random((md.nT, 4)), rng.random(S.n_extra)
    Jg, _ = S.apply(dev(Jin), dev(Bin))
    bg = S.balance(dev(Jin), dev(Bin), Jg)
    _, _, psio = O.apply(Jin, Bin, want_psi=True)
    bo = O.balance(Jin, Bin, psio)
    for k in bo:
        assert abs(bg[k] - bo[k]) < 1e-12 * max(1.0, abs(bo[k]))
    assert abs(bg["emitted"] + bg["incoming"] - bg["absorbed"] - bg["escaped"] - bg["reflective_net"]) < \
        1e-12 * bg["emitted"]


MOMENT_KERNELS = {"tcgen05": tr._lib.TR_MOMENTS_TCGEN05, "mma_sync": tr._lib.TR_MOMENTS_MMA_SYNC,
                  "tma_ffma2": tr._lib.TR_MOMENTS_TMA_FFMA2}


@pytest.mark.parametrize("precision,kernel", [(64, None), (32, "tcgen05"), (32, "mma_sync"), (32, "tma_ffma2")])
def test_moments_match_oracle(cuda, precision, kernel):
    md, ph, S, O = pair(scattering_box(), op.ordinates_product(6, 12))
    if kernel:
        S.set_moments_kernel(MOMENT_KERNELS[kernel])
    S.apply(precision=precision)
    _, _, psio = O.apply(want_psi=True)
    mo = O.moments(psio, 16)
    for nmom in (16, 9, 4, 1, 7):
        mg = host(S.moments(nmom))
        assert rel_err(mg, mo[:nmom]) < (1e-13 if precision == 64 else 2e-5)


@pytest.mark.parametrize("n,polar,azim", [((5, 4, 6), 6, 12),     # 72 ordinates: a part-filled stage
                                          ((12, 12, 12), 14, 22),  # 308: 10 stages a tile, 2-3 tiles a CTA
                                          ((12, 12, 12), 2, 4),    # 8: one part-filled stage
                                          ((6, 6, 6), 32, 32)])    # 1,024: the largest weight table
def test_moments_tcgen05_split_tf32_accuracy(cuda, n, polar, azim):
    """The tensor-core contraction against an FP64 sum over the same FP32 psi
    (the GPU's own, widened exactly): split TF32 with FP32 accumulation stays
    within 3e-6 of the largest moment (a single TF32 product would be ~1e-3).
    The tensor core truncates when it accumulates; the tcgen05 kernel deals
    the ordinate steps over four accumulators summed in FP64, the mma.sync
    kernel (up to 384 ordinates) keeps one, and its truncation bias reaches
    about 4e-6 at 308 ordinates, hence its 1e-5 bound."""
    md, ph, S, O = pair(scattering_box(n=n), op.ordinates_product(polar, azim))
    S.apply(precision=32)
    mo = O.moments(host(S.psi()), 16)
    for nmom in (16, 5):
        mg = host(S.moments(nmom))
        assert rel_err(mg, mo[:nmom]) < 3e-6
    if polar * azim <= 384:
        S.set_moments_kernel(tr._lib.TR_MOMENTS_MMA_SYNC)
        assert rel_err(host(S.moments(16)), mo) < 1e-5
    # FFMA2 form: each FP32 accumulator sums an eighth of the ordinates, the
    # eight partial sums are added in FP64
    S.set_moments_kernel(tr._lib.TR_MOMENTS_TMA_FFMA2)
    for nmom in (16, 5):
        assert rel_err(host(S.moments(nmom)), mo[:nmom]) < 1e-6
    with pytest.raises(tr.TransferError):
        S.set_moments_kernel(7)


def test_gmres_fp64_matches_oracle(cuda):
    md, ph, S, O = pair(scattering_box(albedo=0.9), op.ordinates_product(4, 8))
    J, B, rep = S.solve(tol=1e-11, restart=30)
    Jo, Bo, info = O.solve(method=1, tol=1e-11)
    assert rep.converged and info["converged"]
    assert abs(rep.iterations - info["iterations"]) <= 1
    assert rel_err(host(J), Jo) < 1e-9
    assert rel_err(host(B), Bo) < 1e-9


def test_gmres_with_cycles_matches_oracle(cuda):
    md, ph, S, O = pair(tangled_cube(), op.ordinates_product(4, 8))
    J, B, rep = S.solve(tol=1e-11)
    Jo, Bo, info = O.solve(method=1, tol=1e-11)
    assert rep.converged and rel_err(host(J), Jo) < 1e-9


def test_source_iteration_matches_gmres(cuda):
    md, ph, S, O = pair(scattering_box(n=(3, 3, 3)), op.ordinates_product(4, 8))
    J1, _, r1 = S.solve(tol=1e-12)
    J0, _, r0 = S.solve(method=tr._lib.TR_SWEEP_SOURCE_ITERATION, tol=1e-14, max_iter=3000)
    assert r0.converged and r1.converged
    assert rel_err(host(J0), host(J1)) < 1e-10


def test_mixed_precision_solve(cuda):
    md, ph, S, O = pair(scattering_box(albedo=0.95), op.ordinates_product(4, 8))
    J, B, rep = S.solve(mode=tr.TR_MODE_MIXED, tol=1e-9)
    Jo, Bo, info = O.solve(method=1, tol=1e-12)
    assert rep.converged and rep.residual <= 1e-9 and rep.sweeps_f32 > rep.sweeps_f64
    assert rel_err(host(J), Jo) < 1e-6
    # the FP64 balance of the converged field
    Jout, _ = S.apply(J, B)
    b = S.balance(J, B, Jout)
    assert abs(b["emitted"] + b["incoming"] - b["absorbed"] - b["escaped"]) < 1e-8 * b["emitted"]


@pytest.mark.parametrize("engine", ["cluster", "even_parity"])
def test_dsa_gmres_matches_oracle(cuda, engine):
    """Flexible GMRES with the diffusion correction reaches the oracle's
    fixed point in fewer Krylov steps, one diffusion solve per step, with the
    diffusion CG in one thread-block cluster or on the even-parity context
    (the same diffusion matrix on this box, whose faces are axis-aligned)."""
    L = tr._lib
    md, ph = diffusive_box()
    ords = op.ordinates_product(4, 8)
    S = tr.Sweep(0, md, ords, ph, dsa=True)
    O = op.SweepOracle(md, ords, kappa_abs_volume=ph.kappa_abs_volume, face_bc=ph.face_bc,
                       face_incident=ph.face_incident)
    Jo, Bo, info = O.solve(method=1, tol=1e-11)
    J0, B0, r0 = S.solve(tol=1e-10, max_iter=2000)
    eng = L.TR_SWEEP_DSA_CLUSTER if engine == "cluster" else L.TR_SWEEP_DSA_EVEN_PARITY
    J1, B1, r1 = S.solve(tol=1e-10, precondition=L.TR_SWEEP_PREC_DSA, precond_engine=eng, precond_tol=1e-3)
    assert info["converged"] and r0.converged and r1.converged
    assert r1.residual <= 1e-10 and r1.precond_solves == r1.iterations and r1.precond_iterations > 0
    assert r1.iterations < r0.iterations / 2, (r1.iterations, r0.iterations)
    assert rel_err(host(J1), Jo) < 1e-8 and rel_err(host(B1), Bo) < 1e-8
    assert r0.precond_solves == 0


@pytest.mark.parametrize("which", ["tangled_cube", "scattering_box"])
def test_dsa_with_lagged_and_incident_faces(cuda, which):
    """The correction also reaches lagged inflows (cut dependency cycles)
    and leaves the fixed point unchanged with incident and reflective faces."""
    case = tangled_cube() if which == "tangled_cube" else scattering_box(albedo=0.95)
    md, ph = case
    ords = op.ordinates_product(4, 8)
    S = tr.Sweep(0, md, ords, ph, dsa=True)
    if which == "tangled_cube":
        assert S.n_lag > 0
    O = op.SweepOracle(md, ords, kappa_abs_volume=ph.kappa_abs_volume, face_bc=ph.face_bc,
                       face_incident=ph.face_incident)
    Jo, Bo, info = O.solve(method=1, tol=1e-12)
    for mode in (tr.TR_MODE_FP64, tr.TR_MODE_MIXED):
        J, B, rep = S.solve(mode=mode, tol=1e-11 if mode == tr.TR_MODE_FP64 else 1e-9,
                            precondition=tr._lib.TR_SWEEP_PREC_DSA, precond_tol=1e-4)
        assert rep.converged and rep.precond_solves > 0
        tol = 1e-9 if mode == tr.TR_MODE_FP64 else 1e-6
        assert rel_err(host(J), Jo) < tol and rel_err(host(B), Bo) < tol


def test_dsa_engines_agree(cuda):
    """Both diffusion engines solve the same system to 1e-6: the same Krylov
    steps; the cluster engine's two-level CG (aggregation coarse space) needs
    fewer CG iterations than the even-parity context's Jacobi CG."""
    L = tr._lib
    md, ph = diffusive_box(n=(5, 5, 5))
    S = tr.Sweep(0, md, op.ordinates_product(4, 8), ph, dsa=True)
    kw = dict(tol=1e-10, precondition=L.TR_SWEEP_PREC_DSA, precond_tol=1e-6)
    Jc, _, rc = S.solve(precond_engine=L.TR_SWEEP_DSA_CLUSTER, **kw)
    Je, _, re = S.solve(precond_engine=L.TR_SWEEP_DSA_EVEN_PARITY, **kw)
    assert rc.converged and re.converged
    assert abs(rc.iterations - re.iterations) <= 1
    assert 0 < rc.precond_iterations < re.precond_iterations
    assert rel_err(host(Jc), host(Je)) < 1e-8


def test_dsa_mixed_and_source_iteration(cuda):
    md, ph = diffusive_box(n=(4, 4, 4))
    ords = op.ordinates_product(4, 8)
    S = tr.Sweep(0, md, ords, ph, dsa=True)
    Jg, _, rg = S.solve(tol=1e-11)
    Jm, _, rm = S.solve(mode=tr.TR_MODE_MIXED, tol=1e-9, precondition=tr._lib.TR_SWEEP_PREC_DSA)
    assert rm.converged and rm.residual <= 1e-9 and rm.sweeps_f32 > rm.sweeps_f64
    assert rel_err(host(Jm), host(Jg)) < 1e-7
    SI = tr._lib.TR_SWEEP_SOURCE_ITERATION
    _, _, rs0 = S.solve(method=SI, tol=1e-9, max_iter=100, raise_on_error=False)
    Js, _, rs = S.solve(method=SI, tol=1e-9, max_iter=400, precondition=tr._lib.TR_SWEEP_PREC_DSA,
                        precond_tol=1e-6)
    assert rs.converged and not rs0.converged and rs.iterations < 100
    assert rel_err(host(Js), host(Jg)) < 1e-6


def test_dsa_needs_enable(cuda):
    md, ph = diffusive_box(n=(2, 2, 2))
    S = tr.Sweep(0, md, tr.ordinates_product(2, 4), ph)
    with pytest.raises(tr.TransferError):
        S.solve(precondition=tr._lib.TR_SWEEP_PREC_DSA)
    S2 = tr.Sweep(0, md, tr.ordinates_product(2, 4), ph, dsa=True)
    with pytest.raises(tr.TransferError):
        S2.solve(precondition=tr._lib.TR_SWEEP_PREC_DSA, precond_tol=0.0)
    with pytest.raises(tr.TransferError):
        S2.solve(precondition=7)
    with pytest.raises(tr.TransferError):
        S2.solve(precondition=tr._lib.TR_SWEEP_PREC_DSA, precond_engine=5)


def test_stellar_sphere_sweep_matches_oracle(cuda):
    """Configuration 3's shape at a small size (curved vacuum surface, per-tet
    coefficients, albedo 1/3): one FP64 and one FP32 sweep and the solve."""
    from transfer_b200 import workloads as W
    md, ph, _, _ = W.stellar_sphere(n=10, n_polar=4, n_azim=8)
    md_, ph_, S, O = pair((md, ph), op.ordinates_product(4, 8))
    rng = np.random.default_rng(12)
    Jin = rng.random((md.nT, 4))
    J64, _ = S.apply(dev(Jin), None, precision=64)
    Jo, _ = O.apply(Jin, None)
    assert rel_err(host(J64), Jo) < 1e-12
    J32, _ = S.apply(dev(Jin), None, precision=32)
    assert rel_err(host(J32), Jo) < 2e-5
    J, B, rep = S.solve(tol=1e-11)
    Js, Bs, info = O.solve(method=1, tol=1e-11)
    assert rep.converged and rel_err(host(J), Js) < 1e-9


@pytest.mark.parametrize("precision", [64, 32])
def test_batched_sweep_equals_separate_sweeps(cuda, precision):
    """Problems of different sizes, ordinate sets, boundary kinds (reflective
    inflow, cut cycles) in one launch give exactly the separate sweeps."""
    cases = [(scattering_box(), op.ordinates_product(4, 8)), (tangled_cube(), op.ordinates_product(2, 6)),
             (absorbing_slab(nx=20), op.ordinates_product(6, 12)), (scattering_box(n=(8, 8, 8)), tr.lebedev(17))]
    sweeps = [tr.Sweep(0, md, ords, ph) for (md, ph), ords in cases]
    rng = np.random.default_rng(21)
    Js = [dev(rng.random(4 * S.nT)) for S in sweeps]
    Bs = [dev(rng.random(max(S.n_extra, 1))) for S in sweeps]
    out = tr.sweep_apply_batch(sweeps, precision, Js, Bs)
    for S, J, B, (Jb, Bb) in zip(sweeps, Js, Bs, out):
        Jo, Bo = S.apply(J, B if S.n_extra else None, precision=precision)
        assert torch.equal(Jb, Jo) and torch.equal(Bb, Bo)
    assert sum(S.nq for S in sweeps) > 148   # the batch ran the two-per-SM shape in FP32
    with pytest.raises(tr.TransferError):    # the same problem twice in one batch
        tr.sweep_apply_batch([sweeps[0], sweeps[0]], precision)
    with pytest.raises(tr.TransferError):
        tr.sweep_apply_batch(sweeps[:1], 16)


def test_batched_source_iteration_matches_separate_solves(cuda):
    """The graph-replayed batched source iteration reaches each problem's
    own fixed point (FP64 sweeps; FP32 sweeps to the FP32 floor)."""
    cases = [(scattering_box(), op.ordinates_product(4, 8)), (tangled_cube(), op.ordinates_product(2, 6)),
             (absorbing_slab(nx=20), op.ordinates_product(6, 12))]
    sweeps = [tr.Sweep(0, md, ords, ph) for (md, ph), ords in cases]
    SI = tr._lib.TR_SWEEP_SOURCE_ITERATION
    ref = [S.solve(method=SI, tol=1e-13, max_iter=3000) for S in sweeps]
    out, its, res = tr.sweep_solve_batch(sweeps, 64, tol=1e-13, max_iter=3000)
    assert (its > 0).all() and (res < 1e-13).all()
    for (J, B), (Jr, Br, rep) in zip(out, ref):
        assert rel_err(host(J), host(Jr)) < 1e-11 and rel_err(host(B), host(Br)) < 1e-11
    out32, its32, res32 = tr.sweep_solve_batch(sweeps, 32, tol=1e-6, max_iter=3000)
    assert (its32 > 0).all()
    # FP32 sweeps: 1e-4 of the FP64 fixed point; the tangled cube's inverted
    # elements make some systems ill-conditioned (FP32 sweeps differ by 1e-4)
    for (J, B), (Jr, Br, rep), tol in zip(out32, ref, (1e-4, 2e-3, 1e-4)):
        assert rel_err(host(J), host(Jr)) < tol


def test_batched_source_iteration_in_every_launch_form(cuda):
    """Each launch form of the batched source iteration, set on the first
    sweep only, with the smallest problem first: the graph replays the form
    (and the work-queue ticket) of the first sweep the caller passed, not of
    the largest problem still running."""
    cases = [(absorbing_slab(nx=20), op.ordinates_product(2, 6)), (scattering_box(), op.ordinates_product(4, 8)),
             (scattering_box(n=(8, 8, 8)), op.ordinates_product(4, 8))]
    sweeps = [tr.Sweep(0, md, ords, ph) for (md, ph), ords in cases]
    assert sweeps[0].nT < max(S.nT for S in sweeps)
    SI = tr._lib.TR_SWEEP_SOURCE_ITERATION
    ref = [S.solve(method=SI, tol=1e-12, max_iter=3000) for S in sweeps]
    L_ = tr._lib
    for precision, forms in ((64, [L_.TR_BATCH_STATIC_FULL, L_.TR_BATCH_QUEUE_FULL]),
                             (32, [L_.TR_BATCH_STATIC_FULL, L_.TR_BATCH_QUEUE_FULL, L_.TR_BATCH_STATIC_SMALL,
                                   L_.TR_BATCH_QUEUE_SMALL])):
        for f in forms:
            sweeps[0].set_batch_form(f)
            tol = 1e-12 if precision == 64 else 1e-6
            out, its, res = tr.sweep_solve_batch(sweeps, precision, tol=tol, max_iter=3000)
            assert (its > 0).all(), (precision, f)
            for (J, _), (Jr, _, _) in zip(out, ref):
                assert rel_err(host(J), host(Jr)) < (1e-10 if precision == 64 else 1e-4), (precision, f)


def test_autotune_keeps_results(cuda):
    """Both shapes are timed, the faster kept; FP32 sweeps are bitwise the
    same before and after."""
    md, ph = scattering_box(n=(8, 8, 8))
    S = tr.Sweep(0, md, op.ordinates_product(4, 8), ph)
    J = dev(np.random.default_rng(3).random(4 * S.nT))
    J0, B0 = S.apply(J, None, precision=32)
    shape, ms_full, ms_small = S.autotune()
    assert shape in (0, 1) and ms_full > 0 and ms_small > 0
    assert shape == (1 if ms_small < ms_full else 0)
    J1, B1 = S.apply(J, None, precision=32)
    assert torch.equal(J0, J1) and torch.equal(B0, B1)


def test_set_coefficients_matches_the_oracle(cuda):
    """New sigma_t V, sigma_a V and B on an existing sweep (geometry and
    schedule kept) give the oracle's solution for those coefficients."""
    md, ph = scattering_box()
    ords = op.ordinates_product(4, 8)
    S = tr.Sweep(0, md, ords, ph)
    rng = np.random.default_rng(9)
    kv = md.mesh["kappa_volume"] * rng.uniform(0.5, 2.0, md.nT)
    ka = kv * rng.uniform(0.2, 1.0, md.nT)
    Ip = rng.uniform(0.0, 1.0, md.nT)
    S.set_coefficients(kv, ka, Ip)
    mesh = md.mesh.copy()
    mesh["kappa_volume"] = kv
    mesh["I_p"] = Ip
    md2 = tr.MeshData.from_arrays(tetstart=md.tetstart, tetidx=md.tetidx, tetpos=md.tetpos, facestart=md.facestart,
                                  faceidx=md.faceidx, facepos=md.facepos, mesh=mesh, bnd=md.bnd, coords=md.coords,
                                  regions=md.regions, kappa_abs_volume=ka, face_side=md.face_side)
    O = op.SweepOracle(md2, ords, kappa_abs_volume=ka, face_bc=ph.face_bc, face_incident=ph.face_incident)
    J, B, rep = S.solve(tol=1e-11)
    Jo, Bo, info = O.solve(method=1, tol=1e-11)
    assert rep.converged and rel_err(host(J), Jo) < 1e-9 and rel_err(host(B), Bo) < 1e-9
    with pytest.raises(tr.TransferError):
        S.set_coefficients(kv, kv * 2.0)   # sigma_a > sigma_t


def test_absorbing_slab_matches_e2_on_gpu(cuda):
    md, ph = absorbing_slab(nx=80, ny=4, nz=4)
    S = tr.Sweep(0, md, tr.ordinates_product(16, 16), ph)
    J, B, rep = S.solve(tol=1e-10)
    assert rep.converged
    err = np.abs(host(J) - e2_slab_exact(vertex_x(md), 2.0))
    assert err.max() < 0.025 and err.mean() < 0.003


def test_bad_arguments_are_rejected(cuda):
    md, ph = scattering_box(n=(2, 2, 2))
    S = tr.Sweep(0, md, tr.ordinates_product(2, 4), ph)
    with pytest.raises(tr.TransferError):
        S.apply(precision=16)
    with pytest.raises(tr.TransferError):
        S.solve(restart=0)
    # reflective x faces with an ordinate set that is not mirror symmetric in x
    # (an odd number of azimuths)
    bc = np.where(md.face_side <= 1, tr.TR_BC_REFLECTIVE, tr.TR_BC_VACUUM).astype(np.int32)
    with pytest.raises(tr.TransferError):
        tr.Sweep(0, md, tr.ordinates_product(2, 5), tr.Physics(face_bc=bc))
    # a misaligned device vector
    J = torch.zeros(4 * md.nT + 2, dtype=torch.float64, device="cuda")
    with pytest.raises(tr.TransferError):
        S.apply(J[1:1 + 4 * md.nT])


@pytest.mark.parametrize("precision", [64, 32])
def test_adjoint_gradient_matches_oracle(cuda, precision):
    from sweep_cases import adjoint_box
    md, ph, mask = adjoint_box()
    ords = tr.ordinates_product(4, 8)
    mode = tr.TR_MODE_FP64 if precision == 64 else tr.TR_MODE_MIXED
    F, dsa, dss, rep, rep_a = tr.adjoint_gradient(0, md, ords, ph, mask, precision=precision, mode=mode, tol=1e-11)
    Fo, dsa_o, dss_o = op.sweep_adjoint_gradient(md, ords, ph.kappa_abs_volume, ph.face_bc, ph.face_incident, mask)
    assert rep.converged and rep_a.converged
    assert abs(F - Fo) < 1e-10 * abs(Fo)
    tol = 1e-9 if precision == 64 else 2e-5
    assert rel_err(host(dsa), dsa_o) < tol
    assert rel_err(host(dss), dss_o) < tol


def test_adjoint_gradient_rejects_reflective_faces(cuda):
    md, ph = scattering_box(n=(2, 2, 2))
    ords = tr.ordinates_product(2, 4)
    with pytest.raises(tr.TransferError):
        tr.adjoint_gradient(0, md, ords, ph, (md.face_side == 1).astype(np.int32))


def test_milne_slab_matches_the_analytic_e1_solution(cuda):
    """Configuration 2 at full size: the 8x8x160 Milne-type slab (albedo
    0.999, reflective sides, isotropic inflow at z = 20) with the 110-point
    Lebedev set, solved in FP64 and in mixed precision (FP32 sweeps in FP64
    defect correction) to the FP64 residual 1e-8.  With reflective sides it is
    the 1-D slab whose mean intensity solves the E1 (Peierls) integral
    equation (oracle/slab_analytic.py); J at every cell vertex agrees with it
    to the discretisation error of linear-discontinuous elements at h = 1/8
    mean free path and of the 110-point set (the CPU restatement of the sweep
    gives the same: max 2.1e-3, mean 1.5e-4 of max J).  The mixed solution is
    within 1e-6 of the FP64 one."""
    import slab_analytic as sa
    from transfer_b200 import workloads as W
    md, ph, ords, desc = W.milne_sweep()
    assert len(ords[3]) == 110
    S = tr.Sweep(0, md, ords, ph, dsa=True)
    DSA = tr._lib.TR_SWEEP_PREC_DSA
    J64, _, r64 = S.solve(mode=tr.TR_MODE_FP64, tol=1e-8, restart=40, max_iter=5000, precondition=DSA,
                          precond_tol=1e-2)
    Jmx, _, rmx = S.solve(mode=tr.TR_MODE_MIXED, tol=1e-8, restart=40, max_iter=5000, precondition=DSA,
                          precond_tol=1e-2, inner_tol=1e-4)
    assert r64.converged and rmx.converged
    f, est = sa.slab_reference(a=20.0, albedo=0.999, I0=1.0, n=2000)
    z = md.coords[md.mesh["p"].astype(np.int64)][..., 2]
    Jref = f(z)
    scale = np.abs(Jref).max()
    for J in (host(J64), host(Jmx)):
        err = np.abs(J - Jref) / scale
        assert err.max() < 4e-3 and err.mean() < 4e-4, (err.max(), err.mean())
    assert rel_err(host(Jmx), host(J64)) < 1e-6


def test_frequency_group_equals_its_own_sweep(cuda):
    """A group shares its parent's mesh, ordinates and schedule and has its
    own coefficients: its sweep is exactly the sweep of a problem created with
    those coefficients, and the parent's own sweep is unchanged by it."""
    md, ph = scattering_box()
    ords = op.ordinates_product(4, 8)
    P = tr.Sweep(0, md, ords, ph)
    rng = np.random.default_rng(8)
    kv = md.mesh["kappa_volume"] * rng.uniform(0.5, 3.0, md.nT)
    kav = kv * rng.uniform(0.2, 1.0, md.nT)
    Ip = rng.uniform(0.0, 2.0, md.nT)
    G = P.create_group(kv, kav, Ip)
    R = tr.Sweep(0, md, ords, ph)
    R.set_coefficients(kv, kav, Ip)
    J, B = dev(rng.random(4 * md.nT)), dev(rng.random(P.n_extra))
    Jp0, _ = P.apply(J, B, precision=64)
    for prec in (64, 32):
        Jg, Bg = G.apply(J, B, precision=prec)
        Jr, Br = R.apply(J, B, precision=prec)
        assert torch.equal(Jg, Jr) and torch.equal(Bg, Br)
    Jp1, _ = P.apply(J, B, precision=64)
    assert torch.equal(Jp0, Jp1)
    assert P.device_bytes - G.device_bytes >= 16 * P.nq * P.nT   # the task records are not copied
    with pytest.raises(tr.TransferError):          # a group of a group
        G.create_group(kv)
    assert tr.lib.tr_sweep_destroy(P._h) != tr._lib.TR_OK   # the parent outlives its groups
    G.release_work()
    Jg2, _ = G.apply(J, B, precision=64)            # the work space comes back
    assert torch.equal(Jg2, R.apply(J, B, precision=64)[0])


@pytest.mark.parametrize("precision", [64, 32])
def test_batch_launch_forms_give_identical_results(cuda, precision):
    """Static grid or work queue, full or small shared-memory shape: one
    batched sweep of parents and groups gives the separate sweeps' bits; the
    autotuner times every applicable form and keeps one."""
    cases = [(scattering_box(), op.ordinates_product(4, 8)), (absorbing_slab(nx=20), op.ordinates_product(6, 12)),
             (scattering_box(n=(8, 8, 8)), tr.lebedev(17))]
    sweeps = [tr.Sweep(0, md, ords, ph) for (md, ph), ords in cases]
    rng = np.random.default_rng(9)
    for S, ((md, ph), _) in list(zip(sweeps, cases)):
        for g in range(2):
            kv = md.mesh["kappa_volume"] * 10.0 ** (g / 3.0)
            sweeps.append(S.create_group(kv, None if ph.kappa_abs_volume is None else ph.kappa_abs_volume * 10.0 ** (g / 3.0)))
    Js = [dev(rng.random(4 * S.nT)) for S in sweeps]
    Bs = [dev(rng.random(max(S.n_extra, 1))) for S in sweeps]
    ref = [S.apply(J, B if S.n_extra else None, precision=precision) for S, J, B in zip(sweeps, Js, Bs)]
    L_ = tr._lib
    forms = [L_.TR_BATCH_STATIC_FULL, L_.TR_BATCH_QUEUE_FULL]
    if precision == 32:
        forms += [L_.TR_BATCH_STATIC_SMALL, L_.TR_BATCH_QUEUE_SMALL]
    for f in forms:
        sweeps[0].set_batch_form(f)
        out = tr.sweep_apply_batch(sweeps, precision, Js, Bs)
        for (Jb, Bb), (Jo, Bo) in zip(out, ref):
            assert torch.equal(Jb, Jo) and torch.equal(Bb, Bo), f
    form, ms = tr.sweep_autotune_batch(sweeps, precision)
    assert form in forms and set(ms) == set(forms) and all(v > 0 for v in ms.values())
    out = tr.sweep_apply_batch(sweeps, precision, Js, Bs)
    for (Jb, _), (Jo, _) in zip(out, ref):
        assert torch.equal(Jb, Jo)
    with pytest.raises(tr.TransferError):
        sweeps[0].set_batch_form(4)
