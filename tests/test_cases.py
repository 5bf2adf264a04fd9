"""Host logic of the synthetic case builders (CPU only)."""
import numpy as np

from freecfd_b200 import cases


def test_hypersonic_smooth_state():
    """The vacuum-free start of the hypersonic cylinder: freestream pressure
    and temperature everywhere; zero velocity at the wall radius, the seeded
    freestream velocity beyond wall + width, a monotone blend between."""
    case = cases.hypersonic_case(16, 8)
    n = case.state.shape[0]
    rng = np.random.default_rng(3)
    theta = rng.uniform(0.0, 2.0 * np.pi, n)
    r = np.linspace(0.5, 3.0, n)
    cen = np.stack([r * np.cos(theta), r * np.sin(theta), np.zeros(n)], axis=1)
    W = cases.hypersonic_smooth_state(case, cen, width=2.0)
    assert np.array_equal(W[:, [0, 4]], case.state[:, [0, 4]])
    assert np.all(W[0, 1:4] == 0.0)
    far = r >= 2.5
    assert np.array_equal(W[far, 1:4], case.state[far, 1:4])
    s = W[:, 1] / case.state[:, 1]
    assert np.all(np.diff(s) >= -1e-15) and s.min() >= 0.0 and s.max() <= 1.0 + 1e-15
