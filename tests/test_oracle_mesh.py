"""The oracle-side benchmark meshes (oracle/oracle_mesh.py, used by the CPU
baseline and the reference arm of bench.py so that they do not load the
product library) are the product's meshes: same SplitMix64 jitter, same
Kuhn split, same records and adjacency, value for value."""
import numpy as np
import pytest

import oracle_mesh as om
from transfer_b200 import workloads as W


@pytest.mark.parametrize("name", ["config1", "milne_slab_ref"])
def test_oracle_mesh_equals_product_mesh(name):
    ours, maxk = om.workload(name)
    md, ad, _, desc = W.WORKLOADS[name]()
    assert maxk == desc["maxk"]
    assert (ours.nP, ours.nT, ours.nF) == (md.nP, md.nT, md.nF)
    assert np.array_equal(ours.coords, md.coords)
    assert np.array_equal(ours.regions, md.regions)
    for k in ("tetstart", "tetidx", "tetpos", "facestart", "faceidx", "facepos"):
        assert np.array_equal(getattr(ours, k), getattr(md, k)), k
    assert np.array_equal(ours.mesh["p"], md.mesh["p"])
    assert np.array_equal(ours.mesh["I_p"], md.mesh["I_p"])
    assert np.abs(ours.mesh["kappa_volume"] / md.mesh["kappa_volume"] - 1).max() < 1e-14
    assert np.abs(ours.mesh["s"] - md.mesh["s"]).max() < 1e-15
    assert np.array_equal(ours.bnd["p"][:, :3], md.bnd["p"][:, :3])
    assert np.abs(ours.bnd["s"] - md.bnd["s"]).max() < 1e-15


def test_splitmix64_first_values():
    # SplitMix64 from seed 0: the published first output 0xE220A8397B1DCDAF
    u = om.splitmix64_uniform(0, 1)[0]
    assert u == (0xE220A8397B1DCDAF >> 11) * 2.0 ** -53
