"""The second-order advection term (delta3d_advection.rs) in the oracle (CPU only).

The reference's criterion (tests_delta3d.rs:2132-2193): the centred explicit predictor grows a
four-cell mode (Courant 0.264: x7.4 over 60 steps); with the term the mode no longer grows
(|G|^2 = 1 - C^2 + C^4, x0.13).  The term is off by default.
"""
import golden_cases as G
import numpy as np

from oracle import oracle as O


def advection_only(corrected, amplitude, steps):
    """tests_delta3d.rs:2136-2160: a 2 m/s current with a four-cell mode of `amplitude` m/s, advected
    alone (no projection) for `steps` steps of 33 ms."""
    v = O.OracleVolume(128, 4, 6, 0.25, 1025.0, 9.81)
    if corrected:
        v.enable_advection_correction()
    nx, ny, nz = 128, 4, 6
    u = np.zeros((nz, ny, nx + 1), np.float32)
    i = np.arange(1, nx, dtype=np.float32)
    u[:, :, 1:nx] = np.float32(2.0) + np.float32(amplitude) * np.sin(np.float32(np.pi / 2) * i).astype(np.float32)
    v.set_velocity(u.ravel(), np.zeros(v.nv, np.float32), np.zeros(v.nw, np.float32))
    for _ in range(steps):
        v.advect_for_tests(0.033)
    return v.velocity()[0].reshape(nz, ny, nx + 1)


def growth(corrected, steps):
    """tests_delta3d.rs:2164-2180: amplitude of the difference of two runs, with and without the mode,
    projected on sin/cos(pi i/2) in the middle of the domain."""
    a, b = advection_only(corrected, 1e-3, steps), advection_only(corrected, 0.0, steps)
    nx, j, k = 128, 2, 2
    s = c = 0.0
    for i in range(3 * nx // 8, 5 * nx // 8):
        x = float(a[k, j, i]) - float(b[k, j, i])
        ph = np.pi / 2 * i
        s += x * np.sin(ph)
        c += x * np.cos(ph)
    return float(np.hypot(s, c)) / (1e-3 * (nx / 4) / 2)


def test_second_order_advection_stops_the_ftcs_growth():
    ftcs, corrected = growth(False, 60), growth(True, 60)
    want = G.known_answers()["advection_four_cell_mode"]
    lo, hi = want["ftcs_growth_between"]
    assert lo < ftcs < hi, ftcs
    assert corrected < want["corrected_growth_below"], corrected
