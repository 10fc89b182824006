"""TEST AND MEASUREMENT INFRASTRUCTURE ONLY: the benchmark meshes built on
the oracle side, in numpy, without the product library -- so that the CPU
baseline and the reference arm of bench.py run the same workload as the
product without loading it.

  kuhn(n, box, jitter, seed, region)  seeded Kuhn mesh: an n[0] x n[1] x n[2]
      grid on the box, vertex (i, j, k) -> i + (nx+1)(j + (ny+1) k), interior
      vertices jittered by +-jitter h per axis from SplitMix64(seed) (three
      draws per interior vertex, x then y then z, vertices in index order),
      each hexahedron cut into 6 tetrahedra along its main diagonal, one per
      axis permutation (v0, v0 + e_a, v0 + e_a + e_b, v0 + 1).
  records(coords, tets, regions, kappa, Ip)  the reference's MeshData
      records (MeshData.cpp:13-94): per tet kappa V, I_p and s[j], the area
      normal of the face opposite local vertex j pointing away from it;
      vertex -> tet CSR in (tet, local vertex) order; boundary faces (faces
      of one tet) in (tet, local face) order with that tet's s[j]; vertex ->
      face CSR.
The layouts are the reference's `tetrahedron` (128 B) and `face` (64 B)
records, so oracle_py.Oracle binds the result directly.  The workloads are
restated from the benchmark's description (the same generator the product's
tr_meshdata_kuhn implements); tests/test_oracle_mesh.py checks that both
build the same mesh."""
import numpy as np

TET_DTYPE = np.dtype([("p", "<u4", (4,)), ("kappa_volume", "<f8"), ("I_p", "<f8"), ("s", "<f8", (4, 3))])
FACE_DTYPE = np.dtype([("p", "<u4", (4,)), ("s", "<f8", (3,)), ("pad", "<f8", (3,))])
assert TET_DTYPE.itemsize == 128 and FACE_DTYPE.itemsize == 64

_GAMMA = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64_uniform(seed, count):
    """The first `count` uniforms in [0, 1) of SplitMix64(seed): state +=
    gamma, then the two xor-shift-multiply rounds; uniform = (z >> 11) 2^-53."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + _GAMMA * np.arange(1, count + 1, dtype=np.uint64)
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def kuhn(n, box=(0.0, 1.0, 0.0, 1.0, 0.0, 1.0), jitter=0.0, seed=20261203):
    """(coords [nP][3], tets [nT][4] uint32, centroids [nT][3], vertex side mask [nP])."""
    nx, ny, nz = (int(v) for v in n)
    NX, NY, NZ = nx + 1, ny + 1, nz + 1
    h = np.array([(box[1] - box[0]) / nx, (box[3] - box[2]) / ny, (box[5] - box[4]) / nz])
    k, j, i = np.meshgrid(np.arange(NZ), np.arange(NY), np.arange(NX), indexing="ij")
    i, j, k = i.reshape(-1), j.reshape(-1), k.reshape(-1)
    xyz = np.stack([box[0] + i * h[0], box[2] + j * h[1], box[4] + k * h[2]], axis=1)
    side = ((i == 0) * 1 | (i == NX - 1) * 2 | (j == 0) * 4 | (j == NY - 1) * 8 | (k == 0) * 16 |
            (k == NZ - 1) * 32).astype(np.int32)
    interior = np.flatnonzero(side == 0)
    if jitter > 0 and len(interior):
        u = splitmix64_uniform(seed, 3 * len(interior)).reshape(-1, 3)
        xyz[interior] += (2.0 * u - 1.0) * jitter * h
    stride = np.array([1, NX, NX * NY], dtype=np.int64)
    kk, jj, ii = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    v0 = (ii + NX * (jj + NY * kk)).reshape(-1).astype(np.int64)
    perm = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]
    tets = np.empty((len(v0), 6, 4), dtype=np.int64)
    for q, (a, b, _) in enumerate(perm):
        v1 = v0 + stride[a]
        tets[:, q] = np.stack([v0, v1, v1 + stride[b], v0 + stride.sum()], axis=1)
    tets = tets.reshape(-1, 4)
    cent = xyz[tets].mean(axis=1)
    return xyz, tets.astype(np.uint32), cent, side


def records(coords, tets, regions, kappa, Ip):
    """The reference's MeshData arrays for the mesh (see the module text).
    Returns a namespace with nP, nT, nF, coords, regions, mesh, bnd,
    tetstart/tetidx/tetpos and facestart/faceidx/facepos."""
    coords = np.ascontiguousarray(coords, dtype=np.float64)
    tets = np.ascontiguousarray(tets, dtype=np.int64)
    regions = np.ascontiguousarray(regions, dtype=np.int64)
    kappa, Ip = np.asarray(kappa, dtype=np.float64), np.asarray(Ip, dtype=np.float64)
    nP, nT = len(coords), len(tets)
    P = coords[tets]                                                     # [nT][4][3]
    vol = np.abs(np.einsum("ij,ij->i", P[:, 1] - P[:, 0], np.cross(P[:, 2] - P[:, 0], P[:, 3] - P[:, 0]))) / 6.0
    mesh = np.zeros(nT, dtype=TET_DTYPE)
    mesh["p"] = tets
    mesh["kappa_volume"] = vol * kappa[regions]
    mesh["I_p"] = Ip[regions]
    others = [[k for k in range(4) if k != j] for j in range(4)]
    for j in range(4):
        q = P[:, others[j]]                                              # the face opposite j, in tet order
        nrm = 0.5 * np.cross(q[:, 1] - q[:, 0], q[:, 2] - q[:, 0])
        flip = np.einsum("ij,ij->i", nrm, q[:, 0] - P[:, j]) < 0
        nrm[flip] *= -1.0
        mesh["s"][:, j] = nrm
    # vertex -> tet CSR, (tet, local vertex) order within each vertex
    vflat = tets.reshape(-1)
    order = np.argsort(vflat, kind="stable")
    tetstart = np.zeros(nP + 1, dtype=np.uint32)
    tetstart[1:] = np.cumsum(np.bincount(vflat, minlength=nP))
    tetidx = (order // 4).astype(np.uint32)
    tetpos = (order % 4).astype(np.uint32)
    # boundary faces: the face triples owned by one tet, in (tet, face) order
    faces = np.stack([tets[:, others[j]] for j in range(4)], axis=1)     # [nT][4][3]
    keys = np.sort(faces.reshape(-1, 3), axis=1)
    _, inv, cnt = np.unique(keys, axis=0, return_inverse=True, return_counts=True)
    if cnt.max() > 2:
        raise ValueError("non-manifold mesh: a face shared by more than two tets")
    bmask = cnt[inv.reshape(-1)] == 1
    bt, bj = np.divmod(np.flatnonzero(bmask), 4)
    bnd = np.zeros(len(bt), dtype=FACE_DTYPE)
    bnd["p"][:, :3] = faces[bt, bj]
    bnd["s"] = mesh["s"][bt, bj]
    fflat = bnd["p"][:, :3].astype(np.int64).reshape(-1)
    forder = np.argsort(fflat, kind="stable")
    facestart = np.zeros(nP + 1, dtype=np.uint32)
    facestart[1:] = np.cumsum(np.bincount(fflat, minlength=nP))

    class MeshRecords:
        pass
    m = MeshRecords()
    m.nP, m.nT, m.nF = nP, nT, len(bnd)
    m.coords, m.regions, m.mesh, m.bnd = coords, regions.astype(np.int32), mesh, bnd
    m.tetstart, m.tetidx, m.tetpos = tetstart, tetidx, tetpos
    m.facestart, m.faceidx, m.facepos = facestart, (forder // 3).astype(np.uint32), (forder % 3).astype(np.uint32)
    return m


def workload(name, maxk=None):
    """The reference-runnable benchmark meshes: (records, maxk) for
    config1 (16^3 cube, jitter 0.2h, kappa 1, Ip 1 in r < 0.25 about the
    centre) and milne_slab_ref (8x8x160 slab on [0,1]^2 x [0,20], jitter
    0.15h, kappa 1, Ip 1 for z < 10)."""
    if name == "config1":
        xyz, tets, cent, _ = kuhn((16, 16, 16), jitter=0.2, seed=20261203)
        reg = np.where(((cent - 0.5) ** 2).sum(axis=1) < 0.25 ** 2, 1, 2)
        return records(xyz, tets, reg, [0.0, 1.0, 1.0], [0.0, 1.0, 0.0]), (1 if maxk is None else maxk)
    if name == "milne_slab_ref":
        xyz, tets, cent, _ = kuhn((8, 8, 160), box=(0.0, 1.0, 0.0, 1.0, 0.0, 20.0), jitter=0.15, seed=20261203)
        reg = np.where(cent[:, 2] < 10.0, 1, 2)
        return records(xyz, tets, reg, [0.0, 1.0, 1.0], [0.0, 1.0, 0.0]), (3 if maxk is None else maxk)
    raise KeyError(name)
