"""GPU parity of the operator, right-hand side, BLAS-1 and reductions
(kernels.cu) against the FP64 oracle, through the C ABI.

Tolerances: FP64 results agree with the oracle to 1e-13 of the largest
entry (the assembled operator re-associates the reference's sums); FP32
entry points to 2e-6."""
import numpy as np
import pytest
import torch

import oracle_py as op
import transfer_b200 as tr
from common import c1_mesh, golden_angular, random_vector, rel_err, repad, small_mesh

pytestmark = pytest.mark.gpu


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def host(t):
    return t.detach().cpu().numpy()


def setup(md, ad, **phys):
    physics = tr.Physics(**phys) if phys else None
    ctx = tr.CudaContext(0, md, ad, physics)
    O = op.Oracle(md, ad, **phys)
    assert O.aslm == ctx.aslm
    return ctx, O


KINDS = [tr.TR_OPERATOR_TENSOR, tr.TR_OPERATOR_SIMT]


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("maxk", range(8))
def test_lhs_matches_oracle(cuda, maxk, kind):
    md, ad = small_mesh(), golden_angular(maxk)
    ctx, O = setup(md, ad)
    ctx.set_operator(kind)
    f = random_vector(md.nP, ad.slm, ctx.aslm, seed=maxk)
    Af = ctx.allocVector()
    ctx.computeLhs(dev(f), Af)
    ref = O.lhs(f)
    assert rel_err(host(Af), ref) < 1e-13
    assert np.all(host(Af).reshape(md.nP, -1)[:, ad.slm:] == 0)


@pytest.mark.parametrize("kind", KINDS)
def test_lhs_config1_matches_oracle(cuda, kind):
    md, ad = c1_mesh(), golden_angular(1)
    ctx, O = setup(md, ad)
    ctx.set_operator(kind)
    assert (ctx.nP, ctx.nT, ctx.nF) == (4913, 24576, 3072)
    f = random_vector(md.nP, ad.slm, ctx.aslm, seed=5)
    Af = ctx.allocVector()
    ctx.computeLhs(dev(f), Af)
    assert rel_err(host(Af), O.lhs(f)) < 1e-13


@pytest.mark.parametrize("maxk", [0, 1, 3, 5])
def test_lhs_diag_matches_oracle(cuda, maxk):
    md, ad = small_mesh(), golden_angular(maxk)
    ctx, O = setup(md, ad)
    f = random_vector(md.nP, ad.slm, ctx.aslm, seed=10 + maxk)
    Df = ctx.allocVector()
    ctx.computeLhsDiag(dev(f), Df)
    assert rel_err(host(Df), O.lhs_diag(f)) < 1e-13


@pytest.mark.parametrize("maxk", [1, 2])
def test_rhs_matches_oracle(cuda, maxk):
    md, ad = small_mesh(), golden_angular(maxk)
    ctx, O = setup(md, ad)
    b = ctx.allocVector()
    ctx.computeRhs(b)
    assert rel_err(host(b), O.rhs()) < 1e-15


def test_blas_and_reductions_match_oracle(cuda):
    md, ad = small_mesh(), golden_angular(2)
    ctx, O = setup(md, ad)
    x0 = random_vector(md.nP, ad.slm, ctx.aslm, 1)
    y0 = random_vector(md.nP, ad.slm, ctx.aslm, 2)
    n = len(x0)
    for name, args in (("scale", (0.7,)), ("addProd", (None, -1.3)), ("mulAdd", (0.4, None)),
                       ("mulAddProd", (0.25, None, 3.0))):
        x, y = dev(x0), dev(y0)
        call = [x] + [y if a is None else a for a in args]
        getattr(ctx, name)(*call)
        xr = x0.copy()
        cargs = [xr.ctypes.data] + [y0.ctypes.data if a is None else a for a in args]
        getattr(op.lib, {"scale": "oracle_scale", "addProd": "oracle_add_prod", "mulAdd": "oracle_mul_add",
                         "mulAddProd": "oracle_mul_add_prod"}[name])(n, *cargs)
        assert rel_err(host(x), xr) < 1e-15, name
    assert abs(ctx.dot(dev(x0), dev(y0)) / O.dot(x0, y0) - 1) < 1e-13
    assert abs(ctx.norm(dev(x0)) / O.norm(x0) - 1) < 1e-14
    # padding entries never enter the reductions
    xp = x0.copy().reshape(md.nP, -1)
    xp[:, ad.slm:] = 1e30
    assert abs(ctx.norm(dev(xp.reshape(-1))) / O.norm(x0) - 1) < 1e-14


def test_reductions_are_deterministic(cuda):
    md, ad = c1_mesh(), golden_angular(1)
    ctx, _ = setup(md, ad)
    x = dev(random_vector(md.nP, ad.slm, ctx.aslm, 3))
    a = [ctx.dot(x, x) for _ in range(5)]
    assert len(set(a)) == 1
    Af1, Af2 = ctx.allocVector(), ctx.allocVector()
    ctx.computeLhs(x, Af1)
    ctx.computeLhs(x, Af2)
    assert torch.equal(Af1, Af2)


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("maxk", [1, 3, 5, 7])
def test_f32_entry_points(cuda, maxk, kind):
    md, ad = small_mesh(), golden_angular(maxk)
    ctx, O = setup(md, ad)
    ctx.set_operator(kind)
    f = random_vector(md.nP, ad.slm, ctx.aslm, seed=20 + maxk)
    f32 = repad(f, md.nP, ad.slm, ctx.aslm, ctx.aslm_f32).astype(np.float32)
    Af = ctx.allocVector(torch.float32)
    ctx.computeLhs_f32(dev(f32), Af)
    ref = repad(O.lhs(f), md.nP, ad.slm, ctx.aslm, ctx.aslm_f32)
    assert rel_err(host(Af), ref) < 2e-6
    Df = ctx.allocVector(torch.float32)
    ctx.computeLhsDiag_f32(dev(f32), Df)
    assert rel_err(host(Df), repad(O.lhs_diag(f), md.nP, ad.slm, ctx.aslm, ctx.aslm_f32)) < 2e-6
    b = ctx.allocVector(torch.float32)
    ctx.computeRhs_f32(b)
    assert rel_err(host(b), repad(O.rhs(), md.nP, ad.slm, ctx.aslm, ctx.aslm_f32)) < 1e-6
    d = ctx.dot_f32(dev(f32), dev(f32))
    assert abs(d / O.dot(f, f) - 1) < 1e-6


def test_operator_is_symmetric_positive(cuda):
    md, ad = c1_mesh(), golden_angular(2)
    ctx, _ = setup(md, ad)
    f = dev(random_vector(md.nP, ad.slm, ctx.aslm, 1))
    g = dev(random_vector(md.nP, ad.slm, ctx.aslm, 2))
    Af, Ag = ctx.allocVector(), ctx.allocVector()
    ctx.computeLhs(f, Af)
    ctx.computeLhs(g, Ag)
    gAf, Agf = ctx.dot(g, Af), ctx.dot(Ag, f)
    assert abs(gAf - Agf) < 1e-13 * abs(gAf)
    assert ctx.dot(f, Af) > 0


def test_scattering_extension_matches_oracle(cuda):
    md = small_mesh(albedo=(0.0, 0.9, 0.5))
    ad = golden_angular(2)
    assert md.kappa_abs_volume is not None
    ctx, O = setup(md, ad, kappa_abs_volume=md.kappa_abs_volume)
    f = random_vector(md.nP, ad.slm, ctx.aslm, seed=7)
    Af = ctx.allocVector()
    ctx.computeLhs(dev(f), Af)
    assert rel_err(host(Af), O.lhs(f)) < 1e-13
    Df = ctx.allocVector()
    ctx.computeLhsDiag(dev(f), Df)
    assert rel_err(host(Df), O.lhs_diag(f)) < 1e-13


def test_inflow_extension_matches_oracle(cuda):
    md = small_mesh(Ip=(0.0, 0.0, 0.0))
    ad = golden_angular(2)
    bc = np.where(md.face_side == 5, tr.TR_BC_INCIDENT, tr.TR_BC_VACUUM).astype(np.int32)
    inc = np.where(md.face_side == 5, 2.0, 0.0)
    ctx, O = setup(md, ad, face_bc=bc, face_incident=inc)
    b = ctx.allocVector()
    ctx.computeRhs(b)
    ref = O.rhs()
    assert np.abs(ref).max() > 0
    assert rel_err(host(b), ref) < 1e-14
    f = random_vector(md.nP, ad.slm, ctx.aslm, seed=9)
    Af = ctx.allocVector()
    ctx.computeLhs(dev(f), Af)
    assert rel_err(host(Af), O.lhs(f)) < 1e-13


def test_argument_errors(cuda):
    md, ad = small_mesh(), golden_angular(1)
    ctx, _ = setup(md, ad)
    x = ctx.allocVector()
    with pytest.raises(tr.TransferError) as ei:
        ctx.computeLhs(x, x)
    assert ei.value.status == tr._lib.TR_ERR_INVALID_ARG
    with pytest.raises(tr.TransferError):
        ctx.computeLhs(0, x)
    with pytest.raises(tr.TransferError):
        tr.CudaContext(99, md, ad)
