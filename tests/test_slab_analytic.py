"""CPU checks of the analytic (E1 integral-equation) slab solution that the
Milne-type configuration is compared with (oracle/slab_analytic.py): with no
scattering it is the exact uncollided mean intensity (I0 / 2) E2(a - z);
with scattering it closes the particle balance (incident = absorbed +
reflected + transmitted) and its two grids agree."""
import numpy as np
from scipy.special import expn

import slab_analytic as sa


def test_pure_absorber_is_the_uncollided_e2_solution():
    z, J = sa.slab_mean_intensity(a=5.0, albedo=0.0, I0=2.0, n=400)
    assert np.abs(J - expn(2, 5.0 - z)).max() < 1e-15


def test_scattering_slab_closes_the_balance_and_converges():
    errs = []
    for n in (500, 1000):
        z, J = sa.slab_mean_intensity(a=4.0, albedo=0.9, I0=1.0, n=n)
        b = sa.slab_balance(z, J, 4.0, 0.9)
        errs.append(abs(b["incident"] - b["absorbed"] - b["reflected"] - b["transmitted"]) / b["incident"])
    assert errs[1] < 1e-3 and errs[1] < 0.5 * errs[0]   # first order in h, or better
    J, est = sa.slab_reference(a=4.0, albedo=0.9, n=500)
    assert est < 1e-2
    # the extrapolated solution lies between the boundary value and the deep value
    assert 0.0 < J(0.0) < J(2.0) < J(4.0) < 1.0
