"""Shared helpers of the test suite: standard meshes and conversions."""
import os

import numpy as np

import transfer_b200 as tr

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


def golden_angular(maxk):
    g = golden(f"angular_maxk{maxk}.npz")
    return tr.AngularData(tables={k: g[k] for k in ("slm", "omega", "omega_pos", "Ox", "Oy", "Oz")})


def c1_mesh():
    """Config 1: unit cube, 16^3 Kuhn hexahedra (24,576 tets), interior
    jitter +-0.2h, kappa = 1, emission Ip = 1 inside r < 0.25 about the
    centre, vacuum boundaries."""
    return tr.MeshData.kuhn((16, 16, 16), jitter=0.2, seed=20261203, kappa=[0.0, 1.0, 1.0], Ip=[0.0, 1.0, 0.0],
                            region_kind=1, region_arg=(0.5, 0.5, 0.5, 0.25))


def small_mesh(n=(3, 4, 5), jitter=0.2, seed=11, kappa=(0.0, 2.0, 0.5), Ip=(0.0, 1.0, 0.25), albedo=None):
    return tr.MeshData.kuhn(n, jitter=jitter, seed=seed, kappa=list(kappa), Ip=list(Ip), albedo=albedo,
                            region_kind=1, region_arg=(0.5, 0.5, 0.5, 0.3))


def refrun_mesh(g):
    """Mesh of a refrun_*.npz fixture (same generator arguments)."""
    n = tuple(int(x) for x in g["n"])
    r = 0.25 if n == (16, 16, 16) else 0.3
    return tr.MeshData.kuhn(n, jitter=float(g["jitter"]), seed=int(g["seed"]), kappa=list(g["kappa"]),
                            Ip=list(g["Ip"]), region_kind=1, region_arg=(0.5, 0.5, 0.5, r))


def random_vector(nP, slm, aslm, seed=0, dtype=np.float64):
    rng = np.random.default_rng(seed)
    f = np.zeros((nP, aslm), dtype=dtype)
    f[:, :slm] = rng.standard_normal((nP, slm))
    return f.reshape(-1)


def repad(x, nP, slm, a_from, a_to):
    y = np.zeros((nP, a_to), dtype=x.dtype)
    y[:, :slm] = np.asarray(x).reshape(nP, a_from)[:, :slm]
    return y.reshape(-1)


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
