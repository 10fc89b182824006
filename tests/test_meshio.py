"""Mesh I/O in place of the reference's meshProcessor library: the Netgen
.vol reader (the format of radiation.cfg's meshfile, MeshData.cpp:10) and the
legacy VTK writer with saveVtk's fields (main.cpp:209-216)."""
import numpy as np
import pytest

import transfer_b200 as tr


def kuhn(n=(2, 3, 2)):
    return tr.MeshData.kuhn(n, jitter=0.2, seed=5, kappa=[0.0, 2.0, 0.5], Ip=[0.0, 1.0, 0.1], region_kind=1,
                            region_arg=(0.5, 0.5, 0.5, 0.4))


def write_vol(md, path, gi=False, second_order=False):
    """A .vol file of md (surface elements carry bcnr = box side + 1)."""
    tets = md.mesh["p"].astype(np.int64) + 1
    lines = ["mesh3d", "dimension", "3", "geomtype", "0", ""]
    key = "surfaceelementsgi" if gi else "surfaceelements"
    lines += ["# surfnr bcnr domin domout np p1 p2 p3", key, str(md.nF)]
    for f in range(md.nF):
        p = md.bnd[f]["p"][:3].astype(np.int64) + 1
        extra = " 0 0 0" if gi else ""
        lines.append(f"1 {md.face_side[f] + 1} 1 0 3 {p[0]} {p[1]} {p[2]}{extra}")
    lines += ["", "volumeelements", str(md.nT)]
    for t in range(md.nT):
        if second_order:
            lines.append(f"{md.regions[t]} 10 " + " ".join(str(v) for v in tets[t]) + " 1 1 1 1 1 1")
        else:
            lines.append(f"{md.regions[t]} 4 " + " ".join(str(v) for v in tets[t]))
    lines += ["", "edgesegmentsgi2", "0", "", "points", str(md.nP)]
    lines += [f"{x:.17g} {y:.17g} {z:.17g}" for x, y, z in md.coords]
    lines += ["", "endmesh", ""]
    path.write_text("\n".join(lines))


@pytest.mark.parametrize("gi,second", [(False, False), (True, True)])
def test_vol_reader_matches_the_same_mesh(tmp_path, gi, second):
    md = kuhn()
    f = tmp_path / "m.vol"
    write_vol(md, f, gi=gi, second_order=second)
    mv = tr.MeshData.read_vol(f, kappa=[0.0, 2.0, 0.5], Ip=[0.0, 1.0, 0.1])
    ref = tr.MeshData.from_tets(md.coords, md.mesh["p"], md.regions, kappa=[0.0, 2.0, 0.5], Ip=[0.0, 1.0, 0.1])
    assert (mv.nP, mv.nT, mv.nF) == (ref.nP, ref.nT, ref.nF)
    assert np.array_equal(mv.mesh.view(np.uint8), ref.mesh.view(np.uint8))
    assert np.array_equal(mv.bnd.view(np.uint8), ref.bnd.view(np.uint8))
    assert np.array_equal(mv.regions, md.regions)
    # every boundary face carries its surface element's bc number
    side = {tuple(sorted(md.bnd[f]["p"][:3])): md.face_side[f] + 1 for f in range(md.nF)}
    assert all(mv.face_bcnr[f] == side[tuple(sorted(mv.bnd[f]["p"][:3]))] for f in range(mv.nF))


def test_vol_reader_errors(tmp_path):
    with pytest.raises(tr.TransferError):
        tr.MeshData.read_vol(tmp_path / "missing.vol", kappa=[0.0, 1.0], Ip=[0.0, 1.0])
    bad = tmp_path / "bad.vol"
    bad.write_text("mesh3d\nvolumeelements\n1\n1 4 1 2 3 9\npoints\n4\n0 0 0\n1 0 0\n0 1 0\n0 0 1\nendmesh\n")
    with pytest.raises(tr.TransferError):
        tr.MeshData.read_vol(bad, kappa=[0.0, 1.0], Ip=[0.0, 1.0])


def read_vtk(path):
    """Minimal reader of the legacy binary files written here."""
    data = path.read_bytes()
    pos, out, fields = 0, {}, {}

    def line():
        nonlocal pos
        e = data.index(b"\n", pos)
        s = data[pos:e].decode()
        pos = e + 1
        return s

    def block(count, dt):
        nonlocal pos
        a = np.frombuffer(data, dtype=dt, count=count, offset=pos)
        pos += a.nbytes + 1
        return a

    for _ in range(4):
        line()
    n_pts = int(line().split()[1])
    out["points"] = block(3 * n_pts, ">f8").reshape(-1, 3)
    n_cells = int(line().split()[1])
    out["cells"] = block(5 * n_cells, ">i4").reshape(-1, 5)
    line()
    out["types"] = block(n_cells, ">i4")
    n = None
    while pos < len(data):
        words = line().split()
        if not words:
            continue
        if words[0] in ("CELL_DATA", "POINT_DATA"):
            n = int(words[1])
        elif words[0] == "SCALARS":
            line()
            fields[words[1]] = block(n, ">f8")
        elif words[0] == "VECTORS":
            fields[words[1]] = block(3 * n, ">f8").reshape(n, 3)
        elif words[0] == "TENSORS":
            fields[words[1]] = block(9 * n, ">f8").reshape(n, 3, 3)
    return out, fields


def test_vtk_writer_round_trip(tmp_path):
    md = kuhn()
    rng = np.random.default_rng(0)
    U, T, W = rng.random(md.nP), rng.random((6, md.nP)), rng.random((3, md.nT))
    f = tmp_path / "solution.vtk"
    md.write_vtk(f, point_fields={"U": U, "T": T}, cell_fields={"W": W})
    out, fields = read_vtk(f)
    assert np.array_equal(out["points"], md.coords)
    assert np.array_equal(out["cells"][:, 0], np.full(md.nT, 4)) and np.array_equal(out["types"], np.full(md.nT, 10))
    assert np.array_equal(out["cells"][:, 1:], md.mesh["p"].astype(np.int64))
    assert np.array_equal(fields["U"], U) and np.array_equal(fields["W"], W.T)
    full = np.stack([[T[0], T[1], T[2]], [T[1], T[3], T[4]], [T[2], T[4], T[5]]])  # [3, 3, nP]
    assert np.array_equal(fields["T"], np.moveaxis(full, 2, 0))
