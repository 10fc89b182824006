"""tr_dot_noalloc: the dot product for callers that may not allocate device
memory (a host whose memory pool owns the device, a loop where cudaMalloc
would synchronise the device, or a caller without a tr_ctx).  It keeps its
scratch in one static device array, so these tests check that it agrees
with tr_dot on two calls in a row (the shared scratch left by the first call
must not disturb the second) and with an FP64 NumPy dot of the same data,
that an empty vector gives 0.0, that a call at the largest size its scratch
takes (2048 blocks) is right and leaves the scratch ready for the next call,
and that it rejects sizes beyond its limit.

This file is named to be collected last; it passes alone in a fresh process
and after the other tests."""
import ctypes as C

import numpy as np
import pytest

import transfer_b200 as tr
from common import c1_mesh, golden_angular, random_vector, small_mesh

MAX_ENTRIES = 2048 * 256 * 64


def numpy_dot(x, y, nP, aslm, slm):
    """FP64 dot over lm < slm and the scale of its rounding error (sum |x y|)."""
    a = np.asarray(x).reshape(nP, aslm)[:, :slm]
    b = np.asarray(y).reshape(nP, aslm)[:, :slm]
    return float(np.sum(a * b)), float(np.sum(np.abs(a * b)))


def call(x, y, nP, aslm, slm, out, stream=None):
    return tr.lib.tr_dot_noalloc(C.c_void_p(x), C.c_void_p(y), nP, aslm, slm, C.c_void_p(out), stream)


def test_rejects_sizes_beyond_its_scratch():
    # the size check runs before any CUDA call: no device is needed
    st = call(8, 8, MAX_ENTRIES // 32 + 1, 32, 28, 8)
    assert st == tr._lib.TR_ERR_INVALID_ARG
    assert b"exceeds the maximum" in tr.lib.tr_last_error(None)
    assert call(8, 8, 10, 16, 17, 8) == tr._lib.TR_ERR_INVALID_ARG
    assert call(None, 8, 10, 16, 8, 8) == tr._lib.TR_ERR_INVALID_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("mesh, maxk", [(small_mesh, 2), (c1_mesh, 1), (c1_mesh, 5)])
def test_matches_tr_dot_on_two_calls_in_a_row(cuda, mesh, maxk):
    import torch
    md, ad = mesh(), golden_angular(maxk)
    ctx = tr.CudaContext(0, md, ad)
    nP, aslm, slm = ctx.nP, ctx.aslm, ad.slm
    xs = [random_vector(nP, slm, aslm, seed=s) for s in (31, 32, 33)]
    x0, x1, y = [torch.from_numpy(v).cuda() for v in xs]
    ref = [ctx.dot(x0, y), ctx.dot(x1, y)]
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for i, x in enumerate((x0, x1)):   # two calls in a row, then one sync
        st = call(x.data_ptr(), y.data_ptr(), nP, aslm, slm, out.data_ptr() + 8 * i, stream)
        assert st == tr._lib.TR_OK, tr.lib.tr_last_error(None)
    got = out.cpu().numpy()
    for g, r in zip(got, ref):
        assert abs(g / r - 1) < 1e-13
    for g, x in zip(got, xs[:2]):   # and an FP64 NumPy dot of the same data
        d, scale = numpy_dot(x, xs[2], nP, aslm, slm)
        assert abs(g - d) <= 1e-14 * scale
    # same input again: the same bits (the scratch left by earlier calls is reused)
    st = call(x0.data_ptr(), y.data_ptr(), nP, aslm, slm, out.data_ptr() + 8, stream)
    assert st == tr._lib.TR_OK
    assert out.cpu().numpy()[1] == got[0]
    # padding entries never enter the sum
    xp = xs[0].copy().reshape(nP, aslm)
    xp[:, slm:] = 1e30
    st = call(torch.from_numpy(xp.reshape(-1)).cuda().data_ptr(), y.data_ptr(), nP, aslm, slm, out.data_ptr(),
              stream)
    assert st == tr._lib.TR_OK
    assert out.cpu().numpy()[0] == got[0]
    ctx.close()


@pytest.mark.gpu
def test_rejects_host_memory(cuda):
    import torch
    y = torch.zeros(64, dtype=torch.float64, device="cuda")
    h = np.zeros(64)
    st = call(h.ctypes.data, y.data_ptr(), 4, 16, 15, y.data_ptr())
    assert st == tr._lib.TR_ERR_INVALID_ARG
    assert b"device memory" in tr.lib.tr_last_error(None) or b"CUDA pointer" in tr.lib.tr_last_error(None)


@pytest.mark.gpu
def test_empty_vector_gives_zero(cuda):
    import torch
    x = torch.ones(16, dtype=torch.float64, device="cuda")
    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    st = call(x.data_ptr(), x.data_ptr(), 0, 16, 15, out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert st == tr._lib.TR_OK, tr.lib.tr_last_error(None)
    assert out.cpu().numpy()[0] == 0.0


@pytest.mark.gpu
def test_largest_size_then_a_small_call(cuda):
    """nP * aslm = 33,554,432 (256 MiB per vector) fills all 2048 blocks of the
    scratch; the next, small call must still be right (its ticket was reset)."""
    import torch
    aslm, slm = 32, 28
    nP = MAX_ENTRIES // aslm
    rng = np.random.default_rng(7)
    xh = rng.random(nP * aslm)
    yh = rng.standard_normal(nP * aslm)
    x, y = torch.from_numpy(xh).cuda(), torch.from_numpy(yh).cuda()
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = call(x.data_ptr(), y.data_ptr(), nP, aslm, slm, out.data_ptr(), stream)
    assert st == tr._lib.TR_OK, tr.lib.tr_last_error(None)
    d, scale = numpy_dot(xh, yh, nP, aslm, slm)
    nS = 1000
    st = call(x.data_ptr(), y.data_ptr(), nS, aslm, slm, out.data_ptr() + 8, stream)
    assert st == tr._lib.TR_OK, tr.lib.tr_last_error(None)
    got = out.cpu().numpy()
    assert abs(got[0] - d) <= 1e-14 * scale
    ds, scale_s = numpy_dot(xh[:nS * aslm], yh[:nS * aslm], nS, aslm, slm)
    assert abs(got[1] - ds) <= 1e-14 * scale_s
    del x, y
    torch.cuda.empty_cache()
