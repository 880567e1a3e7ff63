"""The oracle's coupling restatement (coupling.rs:289-330) on the CPU.

`sync_from_rigid` is checked against an independent formulation of the
rotation (the quaternion sandwich q v q*, so agreement is to rounding, 1e-14
relative), `reduce_with_state` against a per-sample loop in sample order
(same additions in the same order, so exact bits).
"""
import numpy as np

import oracle as O
from coupling_scene import cube_samples, interleave, rigid_state
from helpers import assert_bits_equal, oracle_dam_break


def _qmul(a, b):
    w1, x1, y1, z1 = a
    w2, x2, y2, z2 = b
    return np.array([w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2, w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                     w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2, w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2])


def _rotate(q, v):
    qc = np.array([q[0], -q[1], -q[2], -q[3]])
    return _qmul(_qmul(q, np.array([0.0, *v])), qc)[1:]


def _scene():
    box = (0.3, 0.15, 0.2)
    os_ = oracle_dam_break(12, 8, 8, box=box)
    l0, n0 = cube_samples(0.02, 3)
    l1, n1 = cube_samples(0.01, 2)
    body, local, normal = interleave([(l0, n0), (l1, n1)])
    X0 = np.array([[0.07, 0.05, 0.09], [0.2, 0.07, 0.05]])
    base = len(os_)
    for k in range(len(body)):
        os_.push_boundary(X0[body[k]] + local[k], 2e-6, normal[k])
    particle = base + np.arange(len(body), dtype=np.int64)
    o = O.World(os_, O.dam_break_params(materialize=False))
    return o, O.Coupler(o, 2, body, local, normal, particle), X0


def test_sync_matches_quaternion_sandwich():
    o, c, X0 = _scene()
    X, Q, V, W = rigid_state(X0, [(0.0, 0.0, -0.05), (0.1, 0.0, 0.0)], [(0.3, 1.0, 0.2), (0.0, 0.0, 1.0)],
                             [4.0, -2.0], 0.37)
    c.sync_from_rigid(X, Q, V, W)
    x, v = o.x(), o.v()
    for k in range(len(c.body)):
        b, i = c.body[k], c.particle[k]
        r = _rotate(Q[b], c.local[k])
        np.testing.assert_allclose(x[i], X[b] + r, rtol=1e-14, atol=1e-16)
        np.testing.assert_allclose(v[i], V[b] + np.cross(W[b], r), rtol=1e-14, atol=1e-15)


def test_reduce_sums_in_sample_order():
    o, c, X0 = _scene()
    X, Q, V, W = rigid_state(X0, [(0.0, 0.0, -0.05), (0.1, 0.0, 0.0)], [(0.3, 1.0, 0.2), (0.0, 0.0, 1.0)],
                             [4.0, -2.0], 0.0)
    c.sync_from_rigid(X, Q, V, W)
    o.step(1e-4)
    f, t = c.reduce_with_state(X)
    bf, x = o.boundary_force(), o.x()
    ef, et = np.zeros((2, 3)), np.zeros((2, 3))
    for k in range(len(c.body)):
        b, i = c.body[k], c.particle[k]
        fb = bf[i]
        ef[b] = ef[b] + fb
        r = x[i] - X[b]
        et[b] = et[b] + np.array([r[1] * fb[2] - r[2] * fb[1], r[2] * fb[0] - r[0] * fb[2],
                                  r[0] * fb[1] - r[1] * fb[0]])
    assert_bits_equal(f, ef, "force")
    assert_bits_equal(t, et, "torque")
    assert np.abs(f[0]).max() > 0.0
