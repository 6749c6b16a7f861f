"""Host precompute: transmit-arrival distances and angle conversions (known answers from the formulas)."""

from __future__ import annotations

import math

import numpy as np
import pytest

from mach_b200 import geometry, wavefront


def test_plane_projection():
    d = np.array([1.0, 0.0, 0.0])
    pts = np.array([[1.0, 0, 0], [2.0, 1.0, 0], [0.0, 3.0, 0], [-1.0, 0, 0]])
    np.testing.assert_allclose(wavefront.plane(np.zeros(3), pts, d), [1.0, 2.0, 0.0, -1.0])


def test_plane_oblique_and_offset_origin():
    d = np.array([1.0, 1.0, 0.0]) / math.sqrt(2.0)
    pts = np.array([[1.0, 1.0, 0.0], [2.0, 2.0, 0.0], [0.0, 0.0, 0.0]])
    np.testing.assert_allclose(wavefront.plane(np.array([1.0, 1.0, 0.0]), pts, d), [0, math.sqrt(2), -math.sqrt(2)],
                               atol=1e-15)
    d3 = np.ones(3) / math.sqrt(3.0)
    assert float(wavefront.plane(np.zeros(3), np.full(3, math.sqrt(3.0)), d3)) == pytest.approx(3.0)


def test_plane_requires_unit_direction():
    with pytest.raises(ValueError, match="direction must be a unit vector"):
        wavefront.plane(np.zeros(3), np.ones(3), np.array([2.0, 0, 0]))


def test_spherical_focused_and_diverging():
    # focused: transducer 5 behind the focus, point 3 past it -> 5 + 3
    assert float(wavefront.spherical(np.array([0, 0, -5.0]), np.array([0, 0, 3.0]), np.zeros(3))) == pytest.approx(8.0)
    # diverging: virtual source 5 behind the transducer, point 3 in front -> -5 + 8
    assert float(wavefront.spherical(np.zeros(3), np.array([0, 0, 3.0]), np.array([0, 0, -5.0]))) == pytest.approx(3.0)
    # point between origin and focus: 3 - 1
    assert float(wavefront.spherical(np.array([0, 0, -3.0]), np.array([0, 0, -1.0]), np.zeros(3))) == pytest.approx(2.0)


def test_spherical_off_axis():
    o, f, p = np.array([2.0, 0.0, -1.0]), np.array([0.0, 0.0, 2.0]), np.array([1.0, 0.0, 4.0])
    assert float(wavefront.spherical(o, p, f)) == pytest.approx(math.sqrt(13) + math.sqrt(5))


def test_wavefront_torch_matches_numpy():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(0)
    pts = rng.normal(size=(50, 3))
    d = np.array([0.6, 0.0, 0.8])
    a = wavefront.plane(np.zeros(3), pts, d)
    b = wavefront.plane(torch.zeros(3, dtype=torch.float64), torch.as_tensor(pts), torch.as_tensor(d))
    np.testing.assert_allclose(a, b.numpy())
    f = np.array([0.1, -0.2, -1.0])
    np.testing.assert_allclose(wavefront.spherical(np.zeros(3), pts, f),
                               wavefront.spherical(torch.zeros(3, dtype=torch.float64), torch.as_tensor(pts),
                                                   torch.as_tensor(f)).numpy())


def test_ultrasound_angles():
    assert geometry.ultrasound_angles_to_cartesian(0.0, 0.0) == pytest.approx((0.0, 0.0, 1.0))
    assert geometry.ultrasound_angles_to_cartesian(math.pi / 2, 0.0, 2.0) == pytest.approx((2.0, 0.0, 0.0), abs=1e-15)
    assert geometry.ultrasound_angles_to_cartesian(0.0, math.pi / 2, 1.5) == pytest.approx((0.0, 1.5, 0.0), abs=1e-15)
    az, el = np.array([-0.2, 0.0, 0.3]), np.array([0.1, 0.0, -0.4])
    v = geometry.ultrasound_angles_to_cartesian(az, el)
    assert v.shape == (3, 3)
    np.testing.assert_allclose(np.linalg.norm(v, axis=-1), 1.0)
    np.testing.assert_allclose(v[:, 0], np.sin(az))


def test_spherical_to_cartesian():
    x, y, z = geometry.spherical_to_cartesian(math.pi / 4, math.pi / 3, 2.0)
    assert (x, y, z) == pytest.approx((2 * math.sin(math.pi / 4) * 0.5, 2 * math.sin(math.pi / 4) * math.sin(math.pi / 3),
                                       2 * math.cos(math.pi / 4)))


def test_transmit_wave_tables():
    dirs = geometry.ultrasound_angles_to_cartesian(np.deg2rad([-10.0, 0.0, 10.0]), np.zeros(3))
    waves = wavefront.PlaneWaves(np.array([0.0, 0.0, 1e-3]), dirs, time_offset_s=[1e-6, 0.0, 2e-6])
    assert waves.model == 1 and len(waves) == 3 and waves.table.shape == (3, 8)
    np.testing.assert_array_equal(waves.table[:, 0:3], [[0.0, 0.0, 1e-3]] * 3)
    np.testing.assert_array_equal(waves.table[:, 3:6], dirs)
    np.testing.assert_array_equal(waves.table[:, 6], [1e-6, 0.0, 2e-6])
    pts = np.random.default_rng(1).normal(scale=1e-2, size=(20, 3))
    want = np.stack([wavefront.plane([0.0, 0.0, 1e-3], pts, d) / 1540.0 for d in dirs]) + np.array([[1e-6], [0], [2e-6]])
    np.testing.assert_allclose(waves.arrivals(pts, 1540.0), want, rtol=0, atol=1e-18)
    with pytest.raises(ValueError):
        wavefront.PlaneWaves(np.zeros(3), [[0.0, 0.0, 2.0]])
    foci = np.array([[0.0, 0.0, 2e-2], [1e-3, 0.0, -5e-3]])
    sw = wavefront.SphericalWaves(np.zeros(3), foci)
    assert sw.model == 2
    np.testing.assert_allclose(sw.arrivals(pts, 1500.0),
                               np.stack([wavefront.spherical(np.zeros(3), pts, f) / 1500.0 for f in foci]))
