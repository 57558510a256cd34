"""Rounded facet edges: shading_normal_near_edge (optics/raytracer/intersect.rs:196) in the
oracle against the reference's own unit tests (intersect.rs:341-421): disabled at radius
<= 0, continuous across a shared edge (the bisector there), exactly flat far from every
edge, and the documented smoothstep blend in between."""
import numpy as np

CORNER = np.array([[0.0, 1.0, 0.0, 0.0], [1.0, 0.0, 0.0, 0.0]], np.float32)


def test_edge_rounding_disabled_by_default(oracle):
    for radius in (0.0, -1.0, -0.001):
        out = oracle.shading_normal_near_edge(CORNER, [0, 0, 5], 0, [0, 1, 0], radius)
        assert np.array_equal(out, np.array([0, 1, 0], np.float32))


def test_edge_rounding_is_continuous_across_a_shared_edge(oracle):
    a = oracle.shading_normal_near_edge(CORNER, [0, 0, 5], 0, [0, 1, 0], 1.0)
    b = oracle.shading_normal_near_edge(CORNER, [0, 0, 5], 1, [1, 0, 0], 1.0)
    assert np.linalg.norm(a - b) < 1e-5
    assert np.linalg.norm(a - np.array([1, 1, 0]) / np.sqrt(2)) < 1e-5


def test_edge_rounding_leaves_the_interior_exactly_flat(oracle):
    out = oracle.shading_normal_near_edge(CORNER, [-10, 0, 5], 0, [0, 1, 0], 1.0)
    assert np.array_equal(out, np.array([0, 1, 0], np.float32))


def test_edge_rounding_partial_blend_matches_the_smoothstep(oracle):
    d = np.float32(0.5)
    t = np.float32(1.0) - d / np.float32(1.0)
    smooth = t * t * (np.float32(3.0) - np.float32(2.0) * t)
    hn, nn = np.array([0, 1, 0], np.float32), np.array([1, 0, 0], np.float32)
    bis = (hn + nn) / np.linalg.norm(hn + nn)
    want = hn * (1 - smooth) + bis * smooth
    want = want / np.linalg.norm(want)
    out = oracle.shading_normal_near_edge(CORNER, [-0.5, 0, 5], 0, hn, 1.0)
    assert np.linalg.norm(out - want) < 1e-5
