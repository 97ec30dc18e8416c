"""CPU: the exact Sod solution used to measure shock-tube runs, against the published star
state of this problem (Toro, "Riemann Solvers and Numerical Methods for Fluid
Dynamics", 3rd ed., Table 4.3, test 1: p* = 0.30313, u* = 0.92745, rho*L = 0.42632,
rho*R = 0.26557)."""
import math

import numpy as np

from fr_sdg_b200.exact_riemann import sod_exact


def test_sod_regions_at_t_02():
    t = 0.2
    x = np.array([0.1, 0.6, 0.75, 0.9])
    rho = sod_exact(x, t)
    assert rho[0] == 1.0 and rho[3] == 0.125
    assert abs(rho[1] - 0.42632) < 5e-5 and abs(rho[2] - 0.26557) < 5e-5


def test_sod_wave_positions():
    """Rarefaction head at x0 - c_L t, contact at x0 + u* t, shock at x0 + S t."""
    t, g = 0.2, 1.4
    cl = math.sqrt(g)
    head = 0.5 - cl * t
    contact = 0.5 + 0.92745 * t
    x = np.array([head - 1e-3, head + 1e-3, contact - 1e-3, contact + 1e-3])
    rho = sod_exact(x, t)
    assert rho[0] == 1.0 and rho[1] < 1.0            # inside the fan just after its head
    assert abs(rho[2] - 0.42632) < 5e-5 and abs(rho[3] - 0.26557) < 5e-5
    # the fan is monotone
    xf = np.linspace(head, 0.5 + (0.92745 - math.sqrt(g * 0.30313 / 0.42632)) * t, 50)
    assert np.all(np.diff(sod_exact(xf, t)) <= 1e-15)
