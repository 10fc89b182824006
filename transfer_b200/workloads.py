"""Standard synthetic problems (no public dataset is involved; all meshes are
generated, seeded).

  config1      unit cube, 16^3 Kuhn hexahedra (24,576 tets), interior jitter
               +-0.2h, kappa = 1, Ip = 1 inside r < 0.25 about the centre,
               vacuum, maxk = 1 (harmonics up to l = 2; 26-point Lebedev
               precision).  Small enough for the reference's own run.
  milne_slab   box [0,1]^2 x [0,20], 8 x 8 x 160 Kuhn hexahedra (61,440
               tets), jitter +-0.15h, kappa = 1, no internal source,
               isotropic inflow I = 1 through z = 20, vacuum elsewhere,
               maxk = 3 (l <= 6; the 86-point set: the reference's rule
               choice 4 maxk + 2 cannot reach the 110-point set).
  milne_slab_ref
               the same 8 x 8 x 160 slab with the reference's own physics
               (the form its program runs): kappa = 1, emission Ip = 1 in
               the tets whose centroid has z < 10 and 0 above (the
               half-space emission of the reference's Milne problem,
               main.cpp:498-515, with the interface at z = 10), vacuum on
               every face, maxk = 3.  desc["regions"] gives the per-region
               kappa and Ip for a radiation.cfg.
  cube64       unit cube, 64^3 Kuhn hexahedra (1,572,864 tets), kappa per
               tet = exp(0.5 g), g a unit Gaussian random field with
               correlation length 0.1 (random-Fourier-feature sample),
               Ip = 1 in a 0.05-radius ball at (0.2, 0.5, 0.5), maxk = 5
               (l <= 10; 194-point precision).
Each returns (MeshData, AngularData, Physics or None, description dict).
The sweep's problems (milne_sweep, stellar_sphere) return (MeshData,
Physics, ordinates, description dict).
"""
import numpy as np

from .core import AngularData, MeshData, Physics
from ._lib import TR_BC_INCIDENT, TR_BC_VACUUM

SEED = 20261203


def config1(maxk=1, n=16):
    md = MeshData.kuhn((n, n, n), jitter=0.2, seed=SEED, kappa=[0.0, 1.0, 1.0], Ip=[0.0, 1.0, 0.0],
                       region_kind=1, region_arg=(0.5, 0.5, 0.5, 0.25))
    desc = dict(workload="config1", mesh=f"{n}^3 Kuhn cube, jitter 0.2h", maxk=maxk,
                physics="kappa=1, Ip=1 in r<0.25, vacuum", regions={"kappa": [0.0, 1.0, 1.0], "Ip": [0.0, 1.0, 0.0]})
    return md, AngularData(maxk), None, desc


def milne_slab(maxk=3, n=(8, 8, 160), depth=20.0, incident=1.0):
    md = MeshData.kuhn(n, box=(0.0, 1.0, 0.0, 1.0, 0.0, depth), jitter=0.15, seed=SEED, kappa=[0.0, 1.0],
                       Ip=[0.0, 0.0])
    side = md.face_side
    bc = np.where(side == 5, TR_BC_INCIDENT, TR_BC_VACUUM).astype(np.int32)
    inc = np.where(side == 5, float(incident), 0.0)
    phys = Physics(face_bc=bc, face_incident=inc)
    desc = dict(workload="milne_slab", mesh=f"{n[0]}x{n[1]}x{n[2]} Kuhn slab [0,1]^2x[0,{depth:g}], jitter 0.15h",
                maxk=maxk, physics=f"kappa=1, no scattering, isotropic inflow I={incident:g} at z={depth:g}, "
                                   "vacuum elsewhere")
    return md, AngularData(maxk), phys, desc


def milne_slab_ref(maxk=3, n=(8, 8, 160), depth=20.0):
    base = MeshData.kuhn(n, box=(0.0, 1.0, 0.0, 1.0, 0.0, depth), jitter=0.15, seed=SEED, kappa=[0.0, 1.0],
                         Ip=[0.0, 0.0])
    tets = base.mesh["p"]
    zc = base.coords[tets.astype(np.int64)][..., 2].mean(axis=1)
    region = np.where(zc < 0.5 * depth, 1, 2).astype(np.int32)
    kappa, Ip = [0.0, 1.0, 1.0], [0.0, 1.0, 0.0]
    md = MeshData.from_tets(base.coords, tets, region, kappa, Ip)
    desc = dict(workload="milne_slab_ref", mesh=f"{n[0]}x{n[1]}x{n[2]} Kuhn slab [0,1]^2x[0,{depth:g}], jitter 0.15h",
                maxk=maxk, physics=f"kappa=1, Ip=1 for z<{0.5 * depth:g} and 0 above, vacuum on every face "
                                   "(the reference's own boundary and source terms)",
                regions={"kappa": kappa, "Ip": Ip})
    return md, AngularData(maxk), None, desc


def gaussian_random_field(points, corr_len=0.1, modes=512, seed=SEED):
    """Unit-variance Gaussian field with covariance exp(-r^2 / (2 l^2)),
    sampled as sqrt(2/M) sum cos(k.x + phi), k ~ N(0, I / l^2)."""
    rng = np.random.default_rng(seed)
    k = rng.standard_normal((modes, 3)) / corr_len
    phi = rng.uniform(0.0, 2.0 * np.pi, modes)
    out = np.zeros(len(points))
    for c in range(0, modes, 64):
        out += np.cos(points @ k[c:c + 64].T + phi[c:c + 64]).sum(axis=1)
    return out * np.sqrt(2.0 / modes)


def cube64(maxk=5, n=64):
    base = MeshData.kuhn((n, n, n), jitter=0.2, seed=SEED, kappa=[0.0, 1.0], Ip=[0.0, 0.0])
    tets = base.mesh["p"]
    cent = base.coords[tets].mean(axis=1)
    kappa_t = np.exp(0.5 * gaussian_random_field(cent))
    hot = ((cent - np.array([0.2, 0.5, 0.5])) ** 2).sum(axis=1) < 0.05 ** 2
    nT = len(tets)
    kappa = np.concatenate([[0.0], kappa_t])
    Ip = np.concatenate([[0.0], hot.astype(np.float64)])
    md = MeshData.from_tets(base.coords, tets, np.arange(1, nT + 1, dtype=np.int32), kappa, Ip)
    desc = dict(workload="cube64", mesh=f"{n}^3 Kuhn cube, jitter 0.2h", maxk=maxk,
                physics="kappa=exp(0.5 GRF(l=0.1)) per tet, Ip=1 in r<0.05 at (0.2,0.5,0.5), vacuum")
    return md, AngularData(maxk), None, desc


WORKLOADS = {"config1": config1, "milne_slab": milne_slab, "milne_slab_ref": milne_slab_ref, "cube64": cube64}


def _ordinates(lebedev_degree, n_polar, n_azim):
    """The named Lebedev set, or a Gauss-Legendre x azimuth product set when
    n_polar and n_azim are given; returns (ordinates, description)."""
    from .sweep import lebedev, ordinates_product
    if n_polar is not None and n_azim is not None:
        return (ordinates_product(n_polar, n_azim),
                f"{n_polar}x{n_azim} Gauss-Legendre x azimuth product set ({n_polar * n_azim})")
    ords = lebedev(lebedev_degree)
    return ords, f"Lebedev degree {lebedev_degree} ({len(ords[3])} points)"


def milne_sweep(n=(8, 8, 160), depth=20.0, albedo=0.999, incident=1.0, lebedev_degree=17, n_polar=None,
                n_azim=None):
    """The Milne-type slab for the discrete-ordinates sweep: 8 x 8 x 160 Kuhn
    hexahedra on [0,1]^2 x [0,20] (61,440 tets, jitter +-0.15h), sigma_t = 1
    with isotropic scattering of albedo 0.999, reflective x / y faces (an
    infinite slab), vacuum at z = 0, isotropic inflow I = 1 at z = 20.
    Ordinates: the 110-point Lebedev set (degree 17; mirror-symmetric, as the
    reflective walls need), or a product set when n_polar / n_azim are given.
    Returns (MeshData, Physics, ordinates, description)."""
    from ._lib import TR_BC_REFLECTIVE
    md = MeshData.kuhn(n, box=(0.0, 1.0, 0.0, 1.0, 0.0, depth), jitter=0.15, seed=SEED, kappa=[0.0, 1.0],
                       Ip=[0.0, 0.0], albedo=[0.0, albedo])
    side = md.face_side
    bc = np.full(md.nF, TR_BC_VACUUM, dtype=np.int32)
    bc[side <= 3] = TR_BC_REFLECTIVE
    bc[side == 5] = TR_BC_INCIDENT
    phys = Physics(kappa_abs_volume=md.kappa_abs_volume, face_bc=bc, face_incident=np.where(side == 5, incident, 0.0))
    ords, odesc = _ordinates(lebedev_degree, n_polar, n_azim)
    desc = dict(workload="milne_sweep", mesh=f"{n[0]}x{n[1]}x{n[2]} Kuhn slab [0,1]^2x[0,{depth:g}], jitter 0.15h",
                ordinates=odesc,
                physics=f"sigma_t=1, isotropic scattering albedo {albedo:g}, reflective x/y, vacuum z=0, "
                        f"isotropic inflow I={incident:g} at z={depth:g}")
    return md, phys, ords, desc


def stellar_sphere(n=96, lebedev_degree=29, n_polar=None, n_azim=None):
    """The stellar sphere for the discrete-ordinates sweep: a Kuhn grid of
    n^3 hexahedra on [-1,1]^3 (jitter +-0.2h) clipped to the tets whose
    centroid lies in r <= 1 (2,779,622 tets for n = 96), absorption
    kappa(r) = 10 (1 - r^2) + 0.1 and isotropic scattering sigma_s = 0.5 kappa
    per tet (sigma_t = 1.5 kappa, albedo 1/3), source B(r) = (1 - r^2)^4,
    vacuum surface.  Ordinates: the 302-point Lebedev set (degree 29), or a
    product set when n_polar / n_azim are given.
    Returns (MeshData, Physics, ordinates, description)."""
    base = MeshData.kuhn((n, n, n), box=(-1.0, 1.0, -1.0, 1.0, -1.0, 1.0), jitter=0.2, seed=SEED,
                         kappa=[0.0, 1.0], Ip=[0.0, 0.0], ball=(0.0, 0.0, 0.0, 1.0))
    tets = base.mesh["p"]
    cent = base.coords[tets.astype(np.int64)].mean(axis=1)
    r2 = np.minimum((cent ** 2).sum(axis=1), 1.0)
    kappa = 10.0 * (1.0 - r2) + 0.1
    nT = len(tets)
    md = MeshData.from_tets(base.coords, tets, np.arange(1, nT + 1, dtype=np.int32),
                            np.concatenate([[0.0], 1.5 * kappa]), np.concatenate([[0.0], (1.0 - r2) ** 4]),
                            albedo=np.concatenate([[0.0], np.full(nT, 1.0 / 3.0)]))
    phys = Physics(kappa_abs_volume=md.kappa_abs_volume)
    ords, odesc = _ordinates(lebedev_degree, n_polar, n_azim)
    desc = dict(workload="stellar_sphere", mesh=f"{n}^3 Kuhn grid on [-1,1]^3 clipped to r<=1 ({nT} tets), "
                                                "jitter 0.2h",
                ordinates=odesc,
                physics="kappa=10(1-r^2)+0.1, sigma_s=0.5 kappa, B=(1-r^2)^4, vacuum surface")
    return md, phys, ords, desc


def cube64_sweep(n=64, albedo=0.3, degree=23):
    """The adjoint-gradient problem for the discrete-ordinates sweep: the
    cube64 mesh (n^3 Kuhn cube, jitter +-0.2h; 1,572,864 tets for n = 64)
    with sigma_t = exp(0.5 g) per tet (g the unit Gaussian random field of
    cube64), scattering albedo 0.3, B = 1 in the 0.05-radius ball at
    (0.2, 0.5, 0.5), vacuum faces; the 194-point Lebedev set (degree 23).
    The functional is the outflow through the faces at x = 1 (face_mask).
    Returns (MeshData, Physics, ordinates, face_mask, description)."""
    from .sweep import lebedev
    base = MeshData.kuhn((n, n, n), jitter=0.2, seed=SEED, kappa=[0.0, 1.0], Ip=[0.0, 0.0])
    tets = base.mesh["p"]
    cent = base.coords[tets.astype(np.int64)].mean(axis=1)
    sigma_t = np.exp(0.5 * gaussian_random_field(cent))
    hot = ((cent - np.array([0.2, 0.5, 0.5])) ** 2).sum(axis=1) < 0.05 ** 2
    nT = len(tets)
    md = MeshData.from_tets(base.coords, tets, np.arange(1, nT + 1, dtype=np.int32),
                            np.concatenate([[0.0], sigma_t]), np.concatenate([[0.0], hot.astype(np.float64)]),
                            albedo=np.concatenate([[0.0], np.full(nT, float(albedo))]))
    phys = Physics(kappa_abs_volume=md.kappa_abs_volume)
    ords = lebedev(degree)
    fx = md.coords[md.bnd["p"][:, :3].astype(np.int64)][..., 0]
    mask = (fx.min(axis=1) > 1.0 - 1e-9).astype(np.int32)   # faces on x = 1
    desc = dict(workload="cube64_sweep", mesh=f"{n}^3 Kuhn cube, jitter 0.2h ({nT} tets)",
                ordinates=f"Lebedev degree {degree} ({len(ords[3])} points)",
                physics=f"sigma_t=exp(0.5 GRF(l=0.1)) per tet, albedo {albedo:g}, B=1 in r<0.05 at (0.2,0.5,0.5), "
                        "vacuum", functional="outflow through x = 1")
    return md, phys, ords, mask, desc


def cube_batch(count=64, lo=2000, hi=400000, seed=SEED, groups=8):
    """Configuration 4's independent problems for the sweep: `count` jittered
    Kuhn cubes (+-0.2h) with tet counts drawn log-uniformly in [lo, hi]
    (rounded to n^3 hexahedra), per-tet base sigma_t lognormal(0, 1), albedo
    uniform in [0, 0.9] per problem, B = 1 in a random sub-box of edge 0.3,
    vacuum; the 50- or 194-point Lebedev set, drawn per problem.  `groups`
    frequency groups per problem: group g has sigma_t = base x 10^(g/3 - 1)
    with the problem's albedo (no coupling between groups).  Returns
    [(MeshData, Physics, ordinates, group_coefficients)] -- the MeshData and
    Physics carry group 0, group_coefficients lists (sigma_t V, sigma_a V)
    per cell for groups 1 .. groups-1 (tr_sweep_create_group) -- and a
    description."""
    from .sweep import lebedev
    rng = np.random.default_rng(seed)
    sets = {11: lebedev(11), 23: lebedev(23)}
    out = []
    for _ in range(count):
        n = max(2, int(round((np.exp(rng.uniform(np.log(lo), np.log(hi))) / 6.0) ** (1.0 / 3.0))))
        base = MeshData.kuhn((n, n, n), jitter=0.2, seed=int(rng.integers(1 << 30)), kappa=[0.0, 1.0], Ip=[0.0, 0.0])
        tets = base.mesh["p"]
        nT = len(tets)
        cent = base.coords[tets.astype(np.int64)].mean(axis=1)
        c0 = rng.uniform(0.0, 0.7, 3)
        hot = np.all((cent > c0) & (cent < c0 + 0.3), axis=1)
        sigma = rng.lognormal(0.0, 1.0, nT)
        albedo = rng.uniform(0.0, 0.9)
        md = MeshData.from_tets(base.coords, tets, np.arange(1, nT + 1, dtype=np.int32),
                                np.concatenate([[0.0], sigma * 10.0 ** (-1.0)]),
                                np.concatenate([[0.0], hot.astype(np.float64)]),
                                albedo=np.concatenate([[0.0], np.full(nT, albedo)]))
        kv0 = md.mesh["kappa_volume"].copy()
        gc = [(kv0 * 10.0 ** (g / 3.0), kv0 * 10.0 ** (g / 3.0) * (1.0 - albedo)) for g in range(1, groups)]
        out.append((md, Physics(kappa_abs_volume=md.kappa_abs_volume), sets[11 if rng.random() < 0.5 else 23], gc))
    desc = dict(workload="cube_batch", problems=count, groups=groups, tets=f"{lo}-{hi} log-uniform",
                physics="sigma_t lognormal(0,1) x 10^(g/3-1) per tet and group, albedo U[0,0.9] per problem, "
                        "B=1 in a random 0.3 box",
                ordinates="Lebedev 50 or 194 per problem")
    return out, desc


def sweep_work(nT, nq, real_bytes=4):
    """Algorithmic (compulsory) work of one sweep of all ordinates: per
    (cell, ordinate) the 16-byte task record is read and psi (4 reals)
    written; per cell the normals, coefficients and vertex map (16 reals) and
    the scalar-flux source (4 reals) are read once; about 220 flops per
    (cell, ordinate) for the 4x4 system and its solve."""
    return nq * nT * (16 + 4 * real_bytes) + nT * 20 * real_bytes, 220 * nq * nT



def algorithmic_work(md, ad, real_bytes=8):
    """Per operator application: bytes and flops as counted for the roofline:
    read f and write A f (2 * real_bytes per vertex and harmonic), 4 vertex
    indices + kappa per tet (24 B), 3 coordinates per vertex (24 B), 3
    indices per boundary face (12 B); 108 flops per tet and harmonic, the
    angular contraction 2 nnz(omega) per vertex and the boundary term
    6 slm^2 per boundary face."""
    slm = ad.slm
    nnz = int((np.abs(ad.omega) > 1e-14 * np.abs(ad.omega).max()).sum())
    byt = 2 * real_bytes * md.nP * slm + 24 * md.nT + 24 * md.nP + 12 * md.nF
    flops = 108 * md.nT * slm + 2 * nnz * md.nP + 6 * md.nF * slm * slm
    return byt, flops


def cg_iteration_work(md, ad, real_bytes=8):
    """Per CG iteration: the operator application (algorithmic_work) plus the
    vector traffic of the iteration (main.cpp:139-158): x += alpha p (3 vector
    passes), r -= alpha Ap (3), p = z + beta p (3) and Ap read once more for
    <p, Ap> (1), ten passes of real_bytes * nP * slm; 2 flops per entry and
    pass-pair (10 nP slm)."""
    byt, flops = algorithmic_work(md, ad, real_bytes)
    return byt + 10 * real_bytes * md.nP * ad.slm, flops + 10 * md.nP * ad.slm
