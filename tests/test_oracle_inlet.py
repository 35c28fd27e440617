"""The open-x extension of the oracle (no counterpart in the reference, which
is periodic in every direction): a moving-wall bounce-back velocity inlet at
x = 0 and a zero-gradient outflow at x = nx - 1."""

import numpy as np

from oracle import psc_oracle as orc


def test_inlet_delivers_the_prescribed_mass_flux():
    u_in = 0.01
    o = orc.OracleSolver(12, np.zeros((0, 10)), tau=0.8, subsamples=2, static_geometry=True,
                         inlet=(1.0, (u_in, 0.0, 0.0)))
    for _ in range(900):
        o.collide_stream_psc()
    flux = np.mean(o.rho * o.ux)
    assert abs(flux - u_in) <= 1e-4 * u_in
    assert np.abs(o.uy).max() == 0.0 and np.abs(o.uz).max() == 0.0
    # uniform along the channel once the transient has left
    assert np.ptp(o.ux) <= 1e-4 * u_in


def test_open_stream_matches_periodic_stream_inside():
    rng = np.random.default_rng(3)
    f = rng.random((19, 7, 5, 6))
    per = orc.stream_push(f)
    opn = orc.stream_push_open_x(f, 1.02, (0.01, -0.002, 0.003))
    for i in range(19):
        cx = int(orc.C[i][0])
        if cx == 0:
            assert np.array_equal(opn[i], per[i])
        elif cx == 1:
            assert np.array_equal(opn[i, 1:], per[i, 1:])
            corr = orc.inlet_correction(i, 1.02, (0.01, -0.002, 0.003))
            assert np.array_equal(opn[i, 0], f[orc.OPP[i], 0] + corr)
        else:
            assert np.array_equal(opn[i, :-1], per[i, :-1])
            cy, cz = int(orc.C[i][1]), int(orc.C[i][2])
            assert np.array_equal(opn[i, -1], np.roll(f[i, -1], (cy, cz), axis=(0, 1)))


def test_bounce_back_term_sums_to_the_mass_flux():
    # sum over the entering directions of 2 w_i rho (c_i . u) / cs^2 = rho u_x
    rho, u = 1.03, (0.02, 0.004, -0.003)
    s = sum(orc.inlet_correction(i, rho, u) for i in range(19) if orc.C[i][0] == 1)
    assert abs(s - rho * u[0]) <= 1e-15
