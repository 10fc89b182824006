"""Problems of the discrete-ordinates sweep tests (seeded Kuhn meshes).

The reference has no sweep, so these are not its cases: they are the
smallest problems that exercise every branch of the sweep -- vacuum,
incident and reflective faces, scattering, emission, and dependency cycles.
"""
import numpy as np

import transfer_b200 as tr

SEED = 20261203


def absorbing_slab(nx=40, ny=4, nz=4, depth=4.0, a=2.0, jitter=0.15):
    """Purely absorbing slab 0 <= x <= depth (sigma_t = 1), emission B = 1
    for x < a, vacuum at x = 0 and x = depth, reflective y / z faces (an
    infinite slab).  The exact mean intensity is
      x < a : 1 - (E2(x) + E2(a - x)) / 2,     x > a : (E2(x - a) - E2(x)) / 2."""
    md = tr.MeshData.kuhn((nx, ny, nz), box=(0.0, depth, 0.0, 1.0, 0.0, 1.0), jitter=jitter, seed=SEED,
                          kappa=[0.0, 1.0, 1.0], Ip=[0.0, 1.0, 0.0], region_kind=2, region_arg=(a, 0, 0, 0))
    bc = np.where(md.face_side >= 2, tr.TR_BC_REFLECTIVE, tr.TR_BC_VACUUM).astype(np.int32)
    return md, tr.Physics(face_bc=bc, face_incident=np.zeros(md.nF))


def scattering_box(n=(5, 4, 6), jitter=0.2, albedo=0.6, incident=0.7):
    """Box with a scattering sphere (sigma_t 2, albedo as given, B = 1)
    inside a thinner medium (sigma_t 0.5, albedo 0.3, B = 0.25); reflective
    y faces, isotropic inflow at x = 0, vacuum elsewhere."""
    md = tr.MeshData.kuhn(n, jitter=jitter, seed=SEED, kappa=[0.0, 2.0, 0.5], Ip=[0.0, 1.0, 0.25],
                          albedo=[0.0, albedo, 0.3], region_kind=1, region_arg=(0.5, 0.5, 0.5, 0.3))
    side = md.face_side
    bc = np.full(md.nF, tr.TR_BC_VACUUM, dtype=np.int32)
    bc[(side == 2) | (side == 3)] = tr.TR_BC_REFLECTIVE
    bc[side == 0] = tr.TR_BC_INCIDENT
    inc = np.where(side == 0, incident, 0.0)
    return md, tr.Physics(kappa_abs_volume=md.kappa_abs_volume, face_bc=bc, face_incident=inc)


def diffusive_box(n=(6, 6, 6), sigma_t=10.0, albedo=0.995):
    """Optically thick, nearly conservative unit cube (cells about sigma_t / n
    mean free paths across), B = 1, reflective y faces and vacuum elsewhere:
    the regime where unaccelerated iterations stall and the diffusion
    correction pays."""
    md = tr.MeshData.kuhn(n, jitter=0.2, seed=SEED, kappa=[0.0, sigma_t, sigma_t], Ip=[0.0, 1.0, 1.0],
                          albedo=[0.0, albedo, albedo], region_kind=1, region_arg=(0.5, 0.5, 0.5, 0.3))
    bc = np.where((md.face_side == 2) | (md.face_side == 3), tr.TR_BC_REFLECTIVE, tr.TR_BC_VACUUM).astype(np.int32)
    return md, tr.Physics(kappa_abs_volume=md.kappa_abs_volume, face_bc=bc, face_incident=np.zeros(md.nF))


def tangled_cube():
    """6^3 Kuhn cube jittered by +-0.36h: some tetrahedra overlap, and the
    upwind graphs of many ordinates have cycles.  Not a physical mesh (no
    energy balance); it exercises the cycle-cutting schedule, whose levels,
    lag slots and sweeps must match the oracle exactly."""
    md = tr.MeshData.kuhn((6, 6, 6), jitter=0.36, seed=2, kappa=[0.0, 1.0, 1.0], Ip=[0.0, 1.0, 0.0],
                          albedo=[0.0, 0.5, 0.5], region_kind=1, region_arg=(0.5, 0.5, 0.5, 0.3))
    return md, tr.Physics(kappa_abs_volume=md.kappa_abs_volume)


def vertex_x(md):
    """x coordinate of each cell's 4 vertices, [nT][4]."""
    return md.coords[md.mesh["p"].astype(np.int64)][..., 0]


def e2_slab_exact(x, a):
    from scipy.special import expn
    x = np.asarray(x, dtype=np.float64)
    inside = 0.5 * ((1.0 - expn(2, np.maximum(x, 0))) + (1.0 - expn(2, np.maximum(a - x, 0))))
    outside = 0.5 * (expn(2, np.maximum(x - a, 0)) - expn(2, np.maximum(x, 0)))
    return np.where(x < a, inside, outside)


def adjoint_box(n=(4, 3, 3), jitter=0.2):
    """Vacuum box with a scattering, emitting sphere (sigma_t 2, albedo 0.6,
    B = 1) in a thinner scattering medium (sigma_t 0.5, albedo 0.3, B = 0.1)
    and isotropic inflow 0.5 through x = 0; the functional is the outflow
    through the faces at x = 1."""
    md = tr.MeshData.kuhn(n, jitter=jitter, seed=SEED, kappa=[0.0, 2.0, 0.5], Ip=[0.0, 1.0, 0.1],
                          albedo=[0.0, 0.6, 0.3], region_kind=1, region_arg=(0.5, 0.5, 0.5, 0.3))
    side = md.face_side
    bc = np.where(side == 0, tr.TR_BC_INCIDENT, tr.TR_BC_VACUUM).astype(np.int32)
    ph = tr.Physics(kappa_abs_volume=md.kappa_abs_volume, face_bc=bc, face_incident=np.where(side == 0, 0.5, 0.0))
    return md, ph, (side == 1).astype(np.int32)


def perturbed(md, ph, cell, d_sigma_a=0.0, d_sigma_s=0.0):
    """The problem with cell's sigma_a / sigma_s changed (volume fixed)."""
    import oracle_py as op
    V = op.tet_volumes(md)[cell]
    mesh = md.mesh.copy()
    mesh["kappa_volume"][cell] += (d_sigma_a + d_sigma_s) * V
    kav = ph.kappa_abs_volume.copy()
    kav[cell] += d_sigma_a * V

    class _M:
        pass
    m = _M()
    m.nT, m.nF, m.mesh, m.bnd = md.nT, md.nF, mesh, md.bnd
    return m, kav
