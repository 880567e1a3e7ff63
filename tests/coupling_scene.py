"""Rigid sample sets and prescribed rigid motion for the coupling tests.

A body is a set of oriented boundary samples (body-frame offset + outward
normal), as `FluidRigidCoupler::add_sample` (coupling.rs:268-286) records
them. The rigid side is replaced by prescribed motion computed here on the
host, identically for product and oracle, so the tests isolate the fluid side
of `CoupledWcsphWorld::step` (coupling.rs:853-866).
"""
import numpy as np


def cube_samples(half, n):
    """n x n samples on each face of a cube of half-width `half` (body frame),
    normals outward."""
    t = (np.arange(n) + 0.5) / n * 2.0 * half - half
    a, b = np.meshgrid(t, t, indexing="ij")
    a, b = a.reshape(-1), b.reshape(-1)
    local, normal = [], []
    for axis in range(3):
        for sign in (-1.0, 1.0):
            p = np.zeros((a.size, 3))
            p[:, axis] = sign * half
            p[:, (axis + 1) % 3] = a
            p[:, (axis + 2) % 3] = b
            nn = np.zeros((a.size, 3))
            nn[:, axis] = sign
            local.append(p)
            normal.append(nn)
    return np.concatenate(local), np.concatenate(normal)


def ring_samples_2d(radius, n):
    """n samples on a circle in the xy plane, normals outward."""
    th = 2.0 * np.pi * np.arange(n) / n
    local = np.stack([radius * np.cos(th), radius * np.sin(th), np.zeros(n)], 1)
    normal = np.stack([np.cos(th), np.sin(th), np.zeros(n)], 1)
    return local, normal


def interleave(sets):
    """Samples of several bodies in round-robin insertion order: (body, local,
    normal), so a per-body reduction must regroup them."""
    body, local, normal = [], [], []
    m = max(len(s[0]) for s in sets)
    for k in range(m):
        for b, (l, nn) in enumerate(sets):
            if k < len(l):
                body.append(b)
                local.append(l[k])
                normal.append(nn[k])
    return np.array(body, np.int64), np.array(local), np.array(normal)


def axis_angle_quat(axis, angle):
    axis = np.asarray(axis, np.float64)
    axis = axis / np.linalg.norm(axis)
    s = np.sin(0.5 * angle)
    return np.array([np.cos(0.5 * angle), axis[0] * s, axis[1] * s, axis[2] * s])


def rigid_state(x0, v, axis, omega, t):
    """Per-body state (x, q, v, omega) at time t for bodies moving at constant
    velocity and spinning at constant rate about a fixed axis."""
    nb = len(x0)
    X = np.array([np.asarray(x0[b]) + t * np.asarray(v[b]) for b in range(nb)])
    Q = np.array([axis_angle_quat(axis[b], omega[b] * t) for b in range(nb)])
    V = np.array(v, np.float64).reshape(nb, 3)
    W = np.array([omega[b] * np.asarray(axis[b], np.float64) / np.linalg.norm(axis[b]) for b in range(nb)])
    return X, Q, V, W
