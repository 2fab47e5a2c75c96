"""The seeded synthetic workloads: phantom activity maps and event generation (CPU)."""

import math

import numpy as np
import torch

from srf_b200 import synthetic as S


def _act(ph, pts):
    return ph.activity_at(torch.tensor(pts, dtype=torch.float64)).numpy()


def test_standard_phantom_activity():
    ph = S.standard_phantom()
    a = _act(ph, [[0, 0, 0], [50, 0, 0], [150, 0, 0], [0, 0, 60]])
    np.testing.assert_array_equal(a, [1.0, 4.0, 0.0, 0.0])
    assert ph.max_activity == 4.0


def test_large_fov_multi_cylinder_phantom():
    h = 500.0
    ph = S.large_fov_phantom(half_length=h)
    assert len(ph.cylinders) == 11 and not ph.spheres
    hot = [c for c in ph.cylinders if c.activity == 4.0]
    cold = [c for c in ph.cylinders if c.activity == 0.0]
    assert len(hot) == 4 and len(cold) == 4
    pts = [[190, 0, 0],                       # body only
           [-70, 40, 0],                      # 2:1 off-centre cylinder
           [0, 0, 0.9 * h],                   # cold centred cylinder, outer third
           [0, 0, 0.0],                       # body (centre, middle third)
           [0, 0, h + 1.0],                   # beyond the axial end
           [250, 0, 0]]                       # outside the body
    np.testing.assert_array_equal(_act(ph, pts), [1.0, 2.0, 0.25, 1.0, 0.0, 0.0])
    for c in ph.cylinders[3:]:
        z = 0.5 * (c.z_lo + c.z_hi)
        assert _act(ph, [[c.xy[0], c.xy[1], z]])[0] == c.activity
        assert abs(math.hypot(*c.xy) - 120.0) < 1e-9
    assert ph.max_activity == 4.0


def test_generated_events_end_on_crystals():
    wl = S.large_256()
    ph = S.large_fov_phantom(half_length=wl.scanner.axial_length / 2)
    ev = S.generate_events(5000, wl.scanner, ph, seed=3).numpy().astype(np.float64)
    assert ev.shape == (5000, 7)
    for p in (ev[:, 0:3], ev[:, 3:6]):
        r = np.hypot(p[:, 0], p[:, 1])
        np.testing.assert_allclose(r, wl.scanner.inner_radius, rtol=1e-5)
        assert np.all(np.abs(p[:, 2]) <= wl.scanner.axial_length / 2 + 1e-3)
    # same seed, same events
    ev2 = S.generate_events(5000, wl.scanner, ph, seed=3).numpy().astype(np.float64)
    np.testing.assert_array_equal(ev, ev2)
