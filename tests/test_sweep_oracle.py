"""CPU tests of the discrete-ordinates sweep oracle (oracle/sweep_oracle.c)
and of the host side of the sweep's C ABI.

The reference has no sweep, so the oracle's parity is pinned analytically:
the purely absorbing slab's mean intensity against the exact E2 solution
(converging under mesh and angle refinement), the discrete energy balance
(emitted + incoming = absorbed + escaped + reflective, to rounding, for any
single sweep and at convergence), and agreement of GMRES with source
iteration."""
import ctypes as C

import numpy as np
import pytest

import oracle_py as op
import transfer_b200 as tr
from sweep_cases import absorbing_slab, e2_slab_exact, scattering_box, tangled_cube, vertex_x


def test_product_ordinates_match_oracle_and_integrate_exactly():
    x, y, z, w = tr.ordinates_product(6, 8)
    ox, oy, oz, ow = op.ordinates_product(6, 8)
    for a, b in ((x, ox), (y, oy), (z, oz), (w, ow)):
        assert np.abs(a - b).max() < 1e-15
    assert abs(w.sum() - 1.0) < 1e-14
    assert np.abs(x * x + y * y + z * z - 1).max() < 1e-14
    # sphere averages: <z^2> = 1/3, <x^2 y^2> = 1/15, odd moments vanish
    assert abs((w * z * z).sum() - 1 / 3) < 1e-14
    assert abs((w * x * x * y * y).sum() - 1 / 15) < 1e-14
    assert abs((w * x * y * z).sum()) < 1e-15


def test_product_ordinates_rejects_bad_arguments():
    assert tr.lib.tr_ordinates_product(0, 4, None, None, None, None) == tr._lib.TR_ERR_INVALID_ARG


def test_sweep_create_without_device_fails_cleanly():
    md, ph = absorbing_slab(nx=4, ny=2, nz=2)
    x, y, z, w = tr.ordinates_product(2, 4)
    ov = tr._lib.tr_ordinates_view()
    ov.nq, ov.x, ov.y, ov.z, ov.w = len(w), x.ctypes.data, y.ctypes.data, z.ctypes.data, w.ctypes.data
    h = C.c_void_p()
    mv, pv = md.view(), ph.view()
    st = tr.lib.tr_sweep_create(0, C.byref(mv), C.byref(pv), C.byref(ov), C.byref(h))
    import torch
    if not torch.cuda.is_available():
        assert st == tr._lib.TR_ERR_NO_DEVICE and not h.value
    else:
        assert st == 0
        tr.lib.tr_sweep_destroy(h)


def test_absorbing_slab_matches_e2_solution_and_converges():
    errs = []
    for nx, npol in ((20, 8), (40, 8), (80, 16)):
        md, ph = absorbing_slab(nx=nx, ny=2 if nx == 20 else 4, nz=2 if nx == 20 else 4)
        S = op.SweepOracle(md, op.ordinates_product(npol, npol), face_bc=ph.face_bc)
        J, B, info = S.solve(method=1, tol=1e-12, max_iter=300)
        assert info["converged"]
        ex = e2_slab_exact(vertex_x(md), 2.0)
        errs.append((np.abs(J - ex).max(), np.abs(J - ex).mean()))
    # discretisation error: a few percent at 8 cells per mean free path with
    # 64 ordinates, shrinking under refinement in space and angle
    assert errs[0][0] < 0.08 and errs[-1][0] < 0.025
    assert errs[-1][1] < 0.3 * errs[0][1]


def test_energy_balance_single_sweep_and_converged():
    md, ph = scattering_box()
    S = op.SweepOracle(md, op.ordinates_product(4, 8), kappa_abs_volume=ph.kappa_abs_volume, face_bc=ph.face_bc,
                       face_incident=ph.face_incident)
    assert S.n_reflective > 0 and S.n_lag == 0
    rng = np.random.default_rng(1)
    Jin, Bin = rng.random((md.nT, 4)), rng.random(S.nB)
    for J0, B0 in ((None, None), (Jin, Bin)):
        _, _, psi = S.apply(J0, B0, want_psi=True)
        b = S.balance(J0, B0, psi)
        assert abs(b["emitted"] + b["incoming"] - b["absorbed"] - b["escaped"] - b["reflective_net"]) < 1e-13
    J, B, info = S.solve(method=1, tol=1e-12)
    assert info["converged"]
    J2, B2, psi = S.apply(J, B, want_psi=True)
    assert np.abs(J2 - J).max() < 1e-10 and np.abs(B2 - B).max() < 1e-10
    b = S.balance(J, B, psi)
    sav = ph.kappa_abs_volume
    assert abs(b["absorbed"] - (sav * J.mean(axis=1)).sum()) < 1e-10
    assert abs(b["reflective_net"]) < 1e-10
    assert abs(b["emitted"] + b["incoming"] - b["absorbed"] - b["escaped"]) < 1e-12


def test_gmres_and_source_iteration_agree():
    md, ph = scattering_box(n=(3, 3, 3))
    S = op.SweepOracle(md, op.ordinates_product(4, 8), kappa_abs_volume=ph.kappa_abs_volume, face_bc=ph.face_bc,
                       face_incident=ph.face_incident)
    J1, B1, i1 = S.solve(method=1, tol=1e-12)
    J0, B0, i0 = S.solve(method=0, tol=1e-14, max_iter=3000)
    assert i0["converged"] and i1["converged"] and i1["iterations"] < i0["iterations"]
    assert np.abs(J1 - J0).max() < 1e-10


def test_oracle_is_thread_count_independent():
    md, ph = scattering_box(n=(3, 3, 3))
    S = op.SweepOracle(md, op.ordinates_product(4, 8), kappa_abs_volume=ph.kappa_abs_volume, face_bc=ph.face_bc,
                       face_incident=ph.face_incident)
    n0 = op.lib.oracle_num_threads()
    try:
        op.lib.oracle_set_num_threads(1)
        a = S.apply(want_psi=True)
        op.lib.oracle_set_num_threads(max(n0, 4))
        b = S.apply(want_psi=True)
    finally:
        op.lib.oracle_set_num_threads(n0)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_cycle_cutting_schedule():
    md, ph = tangled_cube()
    S = op.SweepOracle(md, op.ordinates_product(4, 8), kappa_abs_volume=ph.kappa_abs_volume)
    assert S.forced > 0 and S.n_lag > 0
    lv = S.levels()
    assert lv.min() == 0 and lv.max() == S.max_levels - 1
    J, B, info = S.solve(method=1, tol=1e-11)
    assert info["converged"]
    J2, B2 = S.apply(J, B)
    assert np.abs(B2 - B).max() < 1e-9 * max(1.0, np.abs(B).max())


def test_moments_l0_is_scalar_flux():
    md, ph = scattering_box(n=(3, 3, 3))
    S = op.SweepOracle(md, op.ordinates_product(6, 12), kappa_abs_volume=ph.kappa_abs_volume, face_bc=ph.face_bc,
                       face_incident=ph.face_incident)
    J, B, psi = S.apply(want_psi=True)
    mom = S.moments(psi, 16)
    assert np.abs(mom[0] - J).max() < 1e-15
    # l = 1 moments are sqrt(3) times the current components <Omega psi>
    x, y, z, w = S.ox, S.oy, S.oz, S.w
    Fx = np.einsum("q,q,qcj->cj", w, x, psi)
    assert np.abs(mom[3] - np.sqrt(3) * Fx).max() < 1e-13


def test_adjoint_gradient_matches_central_differences():
    from sweep_cases import adjoint_box, perturbed
    md, ph, mask = adjoint_box()
    ords = op.ordinates_product(4, 8)
    F, dsa, dss = op.sweep_adjoint_gradient(md, ords, ph.kappa_abs_volume, ph.face_bc, ph.face_incident, mask)
    rng = np.random.default_rng(7)
    for c in rng.choice(md.nT, 6, replace=False):
        for which in ("a", "s"):
            sig = (ph.kappa_abs_volume[c] if which == "a" else md.mesh["kappa_volume"][c] - ph.kappa_abs_volume[c])
            h = 1e-4 * sig / op.tet_volumes(md)[c]
            Fs = []
            for sgn in (1, -1):
                kw = {"d_sigma_a": sgn * h} if which == "a" else {"d_sigma_s": sgn * h}
                m, kav = perturbed(md, ph, c, **kw)
                O = op.SweepOracle(m, ords, kappa_abs_volume=kav, face_bc=ph.face_bc, face_incident=ph.face_incident)
                J, B, info = O.solve(method=1, tol=1e-13)
                _, _, psi = O.apply(J, B, want_psi=True)
                Fs.append(O.outflow(psi, mask))
            fd = (Fs[0] - Fs[1]) / (2 * h)
            g = dsa[c] if which == "a" else dss[c]
            assert abs(g - fd) < 1e-6 * max(abs(fd), 1e-3 * abs(F)), (c, which, g, fd)
