"""TEST INFRASTRUCTURE ONLY: the E1 integral-equation ("analytic") solution
of the plane-parallel slab that the Milne-type configuration reduces to.

Slab 0 <= z <= a (optical depths, sigma_t = 1), isotropic scattering of
albedo c, isotropic incident intensity I0 on the face z = a, vacuum at z = 0.
With reflective side walls the 3-D problem is this 1-D one, and its mean
intensity J(z) = (1/4pi) int I dOmega solves the Peierls equation

    J(z) = (I0 / 2) E2(a - z) + (c / 2) int_0^a E1(|z - z'|) J(z') dz'

(the uncollided mean intensity of the incident beam plus the scattered
contribution through the slab kernel E1 / 2).  It is solved by product
integration: J piecewise constant on n cells, the kernel integrated exactly
over each cell with int_0^d E1 = 1 - E2(d), collocation at the cell centres
(first order in h), and two grids are combined by Richardson extrapolation
(slab_reference).  E_n are scipy's (scipy.special.expn, against which the
oracle's own E_n are checked in tests/test_oracle.py), not the reference's
xE1, whose x > 1 branch returns x e^x E1(x) (E1.cpp:136-160).

The reference's own analytic Milne solution (main.cpp:498-515, soltype 2)
is the pure absorber with half-space emission; with c = 0 and the source
moved to the incident face this solver reduces to the same E2 form."""
import numpy as np
from scipy.special import expn


def _en(n, x):
    return expn(n, np.asarray(x, dtype=np.float64))


def slab_mean_intensity(a=20.0, albedo=0.999, I0=1.0, n=4000):
    """Returns (z_centres, J) of the Peierls solution on n cells."""
    h = a / n
    z = (np.arange(n) + 0.5) * h
    edges = np.arange(n + 1) * h
    # E2 of every centre-to-edge distance, once
    d = np.abs(z[:, None] - edges[None, :])
    E2 = _en(2, d)
    K = np.zeros((n, n))
    # cell j = [edges[j], edges[j+1]]; for z_i outside it the integral of
    # E1(|z_i - z'|) is |E2(d_near) - E2(d_far)|
    K = np.abs(E2[:, :-1] - E2[:, 1:])
    np.fill_diagonal(K, 2.0 * (1.0 - _en(2, np.array([0.5 * h]))[0]))
    S0 = 0.5 * I0 * _en(2, a - z)
    A = np.eye(n) - 0.5 * albedo * K
    return z, np.linalg.solve(A, S0)


def slab_reference(a=20.0, albedo=0.999, I0=1.0, n=4000):
    """J(z) as a callable: the n- and 2n-cell solutions, each interpolated
    linearly, combined as 2 J_2n - J_n (the first-order error cancels; the
    difference of the two grids is returned as the error estimate)."""
    z1, J1 = slab_mean_intensity(a, albedo, I0, n)
    z2, J2 = slab_mean_intensity(a, albedo, I0, 2 * n)

    def J(zq):
        zq = np.clip(np.asarray(zq, dtype=np.float64), 0.0, a)
        return 2.0 * np.interp(zq, z2, J2) - np.interp(zq, z1, J1)
    zs = np.linspace(0.0, a, 2001)
    est = float(np.abs(np.interp(zs, z2, J2) - np.interp(zs, z1, J1)).max() / np.abs(J2).max())
    return J, est


def slab_balance(z, J, a, albedo, I0=1.0):
    """Incident, absorbed, reflected and transmitted flux per unit area of a
    slab solution (mean-intensity units times pi):
    in = pi I0, absorbed = 4 pi (1 - c) int J, reflected (out of z = a) =
    2 pi c int J E2(a - z), transmitted (out of z = 0) = 2 pi c int J E2(z) +
    2 pi I0 E3(a)."""
    h = z[1] - z[0]
    absorbed = 4 * np.pi * (1 - albedo) * J.sum() * h
    reflected = 2 * np.pi * albedo * (J * _en(2, a - z)).sum() * h
    transmitted = 2 * np.pi * albedo * (J * _en(2, z)).sum() * h + 2 * np.pi * I0 * _en(3, np.array([a]))[0]
    return dict(incident=np.pi * I0, absorbed=absorbed, reflected=reflected, transmitted=transmitted)


def interpolate(z, J, zq):
    return np.interp(zq, z, J)
