"""Failure detection without a GPU fault.  The persistent CG kernels meet at a
grid barrier whose waits are bounded (a poll limit, then an error flag that
the host reads).  Here a cooperative grid in which one block never arrives
must give up, report the timeout, and leave the device usable; a grid in
which every block arrives must not."""
import ctypes as C

import pytest
import torch

import transfer_b200 as tr


def run(skip, rounds=8, polls=1 << 14):
    t = C.c_int(-1)
    st = tr.lib.tr_selftest_grid_barrier(0, skip, rounds, polls, C.byref(t))
    assert st == tr._lib.TR_OK, tr.lib.tr_last_error(None)
    return t.value


def test_selftest_rejects_bad_arguments_before_touching_a_device():
    t = C.c_int(-1)
    assert tr.lib.tr_selftest_grid_barrier(0, -1, 0, 16, C.byref(t)) == tr._lib.TR_ERR_INVALID_ARG
    assert tr.lib.tr_selftest_grid_barrier(0, -1, 1, 1 << 25, C.byref(t)) == tr._lib.TR_ERR_INVALID_ARG


@pytest.mark.gpu
def test_barrier_completes_when_every_block_arrives(cuda):
    assert run(-1) == 0


@pytest.mark.gpu
def test_barrier_gives_up_when_a_block_never_arrives(cuda):
    assert run(3) == 1
    assert run(0, rounds=1) == 1
    # the device and this process's context are still usable
    assert run(-1) == 0
    x = torch.ones(4096, dtype=torch.float64, device="cuda")
    assert float(x.sum()) == 4096.0
