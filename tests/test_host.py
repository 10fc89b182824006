"""CPU tests of the product's host side against the reference's own outputs
(golden fixtures from tests/golden/make_golden.py), the C-ABI surface and
host-side error handling.  No GPU needed."""
import ctypes as C
import json
import os
import re

import numpy as np
import pytest

import transfer_b200 as tr
from transfer_b200 import _lib as L
from common import GOLDEN, golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "transfer_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tr_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) > 40
    lib = C.CDLL(tr.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    bound = {p[0] for p in L.PROTOTYPES}
    assert set(names) == bound, set(names) ^ bound


def test_record_layouts_match_reference():
    # tetrahedron.h:20 / face.h:18 compile-time asserts
    assert C.sizeof(L.tr_tetrahedron) == 128 and tr.TET_DTYPE.itemsize == 128
    assert C.sizeof(L.tr_face) == 64 and tr.FACE_DTYPE.itemsize == 64
    assert L.tr_tetrahedron.kappa_volume.offset == 16 and L.tr_tetrahedron.s.offset == 32
    assert L.tr_face.s.offset == 16


def test_abi_version_and_status_strings():
    assert tr.lib.tr_abi_version() == tr._lib.ABI_VERSION == 2
    assert tr.lib.tr_status_string(0) == b"ok"
    assert tr.lib.tr_status_string(3) == b"not converged"


@pytest.mark.parametrize("maxk", range(8))
def test_angular_tables_match_reference(maxk):
    g = golden(f"angular_maxk{maxk}.npz")
    ad = tr.AngularData(maxk)
    assert ad.slm == int(g["slm"]) == (1 + maxk) * (1 + 2 * maxk)
    np.testing.assert_array_equal(ad.omega_pos, g["omega_pos"])
    # exact quadrature here vs Lebedev there: rounding-level agreement
    assert np.abs(ad.omega - g["omega"]).max() < 1e-12
    for n in ("Ox", "Oy", "Oz"):
        assert np.abs(getattr(ad, n) - g[n]).max() < 1e-12
    assert abs(ad.Ox[0, 0] - 0.5) < 1e-14


def test_angular_rejects_bad_maxk():
    with pytest.raises(tr.TransferError):
        tr.AngularData(8)
    with pytest.raises(tr.TransferError):
        tr.AngularData(-1)


def test_spherical_matches_reference():
    g = golden("misc.npz")
    L_ = int(g["sph_L"])
    x, y, z = g["sph_xyz"]
    vals = g["sph_vals"]
    row = 0
    for l in range(L_ + 1):
        for m in range(-l, l + 1):
            ours = np.array([tr.lib.tr_spherical_value(l, m, x[p], y[p], z[p]) for p in range(len(x))])
            scale = max(1.0, np.abs(vals[row]).max())
            # the reference runs Horner on monomial Legendre coefficients
            # (Spherical.cpp:6-37), which loses ~1e-12 by l = 14
            assert np.abs(ours - vals[row]).max() < 1e-11 * scale, (l, m)
            row += 1


def rule(fn, deg):
    n = fn(deg, None, None, None, None, 0)
    if n < 0:
        return None
    a = np.zeros((4, n))
    assert fn(deg, *(r.ctypes.data for r in a), n) == n
    return a


@pytest.mark.parametrize("deg", [1, 5, 9, 13, 17, 21, 25, 29])
def test_hemiquad_matches_reference(deg):
    g = golden("quadrature.npz")[f"hemi_{deg}"]
    ours = rule(tr.lib.tr_hemiquad, deg)
    assert ours.shape == g.shape
    assert np.abs(ours - g).max() < 1e-14
    assert abs(ours[3].sum() - 1.0) < 1e-14


def _sorted_rule(r):
    r = np.asarray(r)
    idx = np.lexsort((r[2].round(9), r[1].round(9), r[0].round(9)))
    return r[:, idx]


@pytest.mark.parametrize("deg", [2, 6, 10, 13, 14, 17, 18, 22, 25, 26, 29, 30])
def test_lebedev_matches_reference(deg):
    """The generated rules are the reference's LebedevQuad point sets
    (LebedevQuad.cpp) up to the order of the points: every rule up to 350
    points (precision 31), the ones with negative orbit weights included
    (74, 230 and 266 points)."""
    g = golden("quadrature.npz")[f"lebedev_{deg}"]
    ours = rule(tr.lib.tr_lebedev, deg)
    assert ours.shape == g.shape
    assert np.abs(_sorted_rule(ours) - _sorted_rule(g)).max() < 1e-11
    assert abs(ours[3].sum() - 1.0) < 1e-14
    # exact for the real harmonics up to the rule's precision
    prec = {6: 3, 26: 7, 50: 11, 74: 13, 86: 15, 110: 17, 146: 19, 194: 23, 230: 25, 266: 27, 302: 29,
            350: 31}[g.shape[1]]
    x, y, z, w = ours
    for l in range(1, prec + 1):
        for m in range(-l, l + 1):
            v = np.array([tr.lib.tr_spherical_value(l, m, a, b, c) for a, b, c in zip(x, y, z)])
            assert abs((w * v).sum()) <= 1e-13 * (np.abs(v).max() * len(v) + 1.0)


@pytest.mark.parametrize("deg", [32, 35, 41])
def test_lebedev_beyond_generated_rules_is_refused(deg):
    assert tr.lib.tr_lebedev(deg, None, None, None, None, 0) == -1


def test_trieig_matches_reference():
    g = golden("misc.npz")
    o = 0
    for n, lm in zip(g["trieig_n"], g["trieig_l"]):
        a, b = g["trieig_a"][o:o + n], g["trieig_b"][o:o + n]
        o += n
        assert abs(tr.trieig(a, b) - lm) <= 1e-12 * abs(lm)


# ---------------------------------------------------------------- Config
CONFIG_CASES = json.load(open(os.path.join(GOLDEN, "configs.json")))


@pytest.mark.parametrize("name", sorted(CONFIG_CASES))
def test_config_matches_reference(name):
    exp = CONFIG_CASES[name]
    path = os.path.join(GOLDEN, f"cfg_{name}.cfg")
    if exp["returncode"] != 0:
        with pytest.raises(tr.TransferError) as ei:
            tr.Config(path)
        assert ei.value.status == L.TR_ERR_CONFIG
        return
    cfg = tr.Config(path)
    res = exp["result"]
    m = dict(kv.split("=") for kv in res[0].split())
    assert cfg.getMaxK() == int(m["maxk"])
    assert cfg.getDevice() == int(m["device"])
    assert cfg.doDump() == bool(int(m["dump"]))
    assert cfg.usePrec() == bool(int(m["prec"]))
    assert cfg.solType() == int(m["soltype"])
    assert cfg.getMeshFilename() == res[1][len("meshfile="):]
    assert cfg.getOutFilename() == res[2][len("outfile="):]
    for line in res[3:]:
        d = dict(kv.split("=") for kv in line.split())
        r = int(d["region"])
        if r > cfg.numRegions():
            continue  # the reference reads uninitialised memory there
        assert cfg.getKappa(r) == float(d["kappa"])
        assert cfg.getIp(r) == float(d["Ip"])


def test_config_additive_keys(tmp_path):
    p = tmp_path / "x.cfg"
    p.write_text("numregs = 1\nangorder = 3\ntolerance = 1e-9\nmode = mixed\n[region 1]\nkappa = 2\nIp = 1\n"
                 "albedo = 0.999\n")
    cfg = tr.Config(p)
    assert cfg.get("tolerance") == "1e-9" and cfg.get("mode") == "mixed"
    assert cfg.region(1, "albedo") == 0.999
    assert cfg.usePrec() is False and cfg.solType() == 0   # defaults instead of garbage


@pytest.mark.parametrize("text,key,line", [
    ("numregs = 1\n[region 1]\nkappa = x\n", "kappa", 3),
    ("numregs = 1\nkappa = 1\n", "kappa", 2),
    ("numregs = 1\n[region 1]\nangorder = 2\n", "angorder", 3),
    ("# c\n[region 1]\n", "numregs", 2),
    ("numregs = 2\n[region 3]\n", "region 3", 2),
    ("numregs = -4\n", "numregs", 1),
])
def test_config_error_names_key_and_line(tmp_path, text, key, line):
    p = tmp_path / "bad.cfg"
    p.write_text(text)
    with pytest.raises(tr.TransferError) as ei:
        tr.Config(p)
    assert ei.value.status == L.TR_ERR_CONFIG
    msg = str(ei.value)
    assert key in msg and f"line {line}" in msg, msg


def test_config_missing_file():
    with pytest.raises(tr.TransferError) as ei:
        tr.Config("/nonexistent/radiation.cfg")
    assert ei.value.status == L.TR_ERR_CONFIG


# -------------------------------------------------------------- MeshData
@pytest.mark.parametrize("name", ["small_k1", "small_k2", "small_k1_prec"])
def test_meshdata_matches_reference(name):
    """The reference's MeshData.cpp built these records from the same mesh."""
    g = golden(f"meshdata_{name}.npz")
    r = golden(f"refrun_{name}.npz")
    md = tr.MeshData.from_tets(g["coords"], g["tets"], g["regions"], list(r["kappa"]), list(r["Ip"]))
    for k in ("tetstart", "tetidx", "tetpos", "facestart", "faceidx", "facepos"):
        np.testing.assert_array_equal(getattr(md, k), g[k], err_msg=k)
    ref_t = g["mesh"].view(tr.TET_DTYPE)
    np.testing.assert_array_equal(md.mesh["p"], ref_t["p"])
    np.testing.assert_array_equal(md.mesh["I_p"], ref_t["I_p"])
    assert np.abs(md.mesh["kappa_volume"] / ref_t["kappa_volume"] - 1).max() < 1e-13
    assert np.abs(md.mesh["s"] - ref_t["s"]).max() < 1e-15
    ref_f = g["bnd"].view(tr.FACE_DTYPE)
    np.testing.assert_array_equal(md.bnd["p"][:, :3], ref_f["p"][:, :3])
    assert np.abs(md.bnd["s"] - ref_f["s"]).max() < 1e-15


def test_kuhn_mesh_config1_sizes():
    md = tr.MeshData.kuhn((16, 16, 16), jitter=0.2, kappa=[0, 1.0], Ip=[0, 1.0])
    assert (md.nP, md.nT, md.nF) == (4913, 24576, 3072)
    assert np.abs(md.mesh["s"].sum(axis=1)).max() < 1e-15          # closure, MeshData.cpp:74-76
    vol = md.mesh["kappa_volume"]                                    # kappa = 1
    assert abs(vol.sum() - 1.0) < 1e-12 and vol.min() > 0
    assert np.all(np.bincount(md.face_side, minlength=6) == 512)
    # interior vertices jittered by at most 0.2 h, boundary vertices fixed
    h = 1 / 16
    ijk = np.stack(np.meshgrid(np.arange(17), np.arange(17), np.arange(17), indexing="ij"), -1)
    lattice = ijk.transpose(2, 1, 0, 3).reshape(-1, 3) * h
    d = np.abs(md.coords - lattice)
    assert d.max() <= 0.2 * h + 1e-15
    onb = (ijk.transpose(2, 1, 0, 3).reshape(-1, 3) % 16 == 0).any(axis=1)
    assert d[onb].max() == 0.0
    md2 = tr.MeshData.kuhn((16, 16, 16), jitter=0.2, kappa=[0, 1.0], Ip=[0, 1.0])
    np.testing.assert_array_equal(md.coords, md2.coords)


def test_kuhn_ball_and_regions():
    md = tr.MeshData.kuhn((12, 12, 12), box=(-1, 1, -1, 1, -1, 1), jitter=0.1, kappa=[0, 1.0, 2.0],
                          Ip=[0, 1.0, 0.0], region_kind=1, region_arg=(0, 0, 0, 0.5), ball=(0, 0, 0, 1.0))
    c = md.coords
    assert np.sqrt((c ** 2).sum(1)).max() < 1.2
    assert set(np.unique(md.regions)) == {1, 2}
    assert np.abs(md.mesh["s"].sum(axis=1)).max() < 1e-15


def test_meshdata_rejects_bad_input():
    xyz = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=float)
    with pytest.raises(tr.TransferError):   # vertex index out of range
        tr.MeshData.from_tets(xyz, [[0, 1, 2, 7]], [1], [0, 1.0], [0, 1.0])
    with pytest.raises(tr.TransferError):   # degenerate tet
        tr.MeshData.from_tets(xyz, [[0, 1, 2, 2]], [1], [0, 1.0], [0, 1.0])
    with pytest.raises(tr.TransferError):   # region out of range
        tr.MeshData.from_tets(xyz, [[0, 1, 2, 3]], [3], [0, 1.0], [0, 1.0])


# --------------------------------------------------- context validation
def _ctx_status(md, ad, device=0):
    mv, av = md.view(), ad.view()
    h = C.c_void_p()
    return tr.lib.tr_ctx_create(device, C.byref(mv), C.byref(av), C.byref(h)), h


def test_ctx_create_rejects_corrupt_mesh_before_touching_a_device():
    md = tr.MeshData.kuhn((2, 2, 2), kappa=[0, 1.0], Ip=[0, 1.0])
    ad = tr.AngularData(1)
    md.tetidx[3] = md.nT + 5
    st, _ = _ctx_status(md, ad)
    assert st == L.TR_ERR_MESH and b"tetidx" in tr.lib.tr_last_error(None)
    md = tr.MeshData.kuhn((2, 2, 2), kappa=[0, 1.0], Ip=[0, 1.0])
    md.mesh["kappa_volume"][0] = -1.0
    st, _ = _ctx_status(md, ad)
    assert st == L.TR_ERR_MESH
    md = tr.MeshData.kuhn((2, 2, 2), kappa=[0, 1.0], Ip=[0, 1.0])
    md.tetpos[0] = (md.tetpos[0] + 1) % 4
    st, _ = _ctx_status(md, ad)
    assert st == L.TR_ERR_MESH
    bad = tr.AngularData(tables=dict(slm=7, omega=np.zeros(147), omega_pos=np.zeros(147, np.uint32),
                                     Ox=np.zeros(49), Oy=np.zeros(49), Oz=np.zeros(49)))
    md = tr.MeshData.kuhn((2, 2, 2), kappa=[0, 1.0], Ip=[0, 1.0])
    st, _ = _ctx_status(md, bad)
    assert st == L.TR_ERR_MESH
    h = C.c_void_p()
    assert tr.lib.tr_ctx_create(0, None, None, C.byref(h)) == L.TR_ERR_MESH
    assert tr.lib.tr_ctx_create(0, C.byref(md.view()), C.byref(ad.view()), None) == L.TR_ERR_INVALID_ARG


def test_calls_on_null_context_fail_cleanly():
    out = C.c_double()
    assert tr.lib.tr_compute_lhs(None, None, None) == L.TR_ERR_INVALID_ARG
    assert tr.lib.tr_dot(None, None, None, C.byref(out)) == L.TR_ERR_INVALID_ARG
    assert tr.lib.tr_ctx_destroy(None) == L.TR_OK


def test_no_cpu_fallback_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    md = tr.MeshData.kuhn((2, 2, 2), kappa=[0, 1.0], Ip=[0, 1.0])
    st, _ = _ctx_status(md, tr.AngularData(1))
    assert st == L.TR_ERR_NO_DEVICE
    with pytest.raises(tr.TransferError):
        tr.CudaContext(0, md, tr.AngularData(1))
