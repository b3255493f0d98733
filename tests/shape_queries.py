"""Seeded queries of the procedural primitive tests (bilinear patches and analytic shapes), in
the layouts of rp_cuda_probe_bilinear / rp_cuda_probe_analytic, shared by the CPU pins and the
GPU parity tests."""

import numpy as np

from rypath_b200 import abi


def bilinear_queries(n=20000, seed=11):
    """Warped, planar and nearly degenerate patches; rays aimed at points of the patch's
    parameter square (and a little outside it), at its edges and corners, from inside and
    outside, with finite and infinite t_max."""
    rng = np.random.default_rng(seed)
    q = np.zeros((n, 20), np.float32)
    for i in range(n):
        kind = i % 5
        p = rng.uniform(-1, 1, (4, 3))
        if kind == 1:  # planar: p11 = p10 + p01 - p00
            p[3] = p[1] + p[2] - p[0]
        elif kind == 2:  # a thin sliver
            p[2] = p[0] + 1e-3 * rng.normal(size=3)
        elif kind == 3:  # large coordinates, small patch
            p = 100.0 + 0.01 * p
        u, v = rng.uniform(-0.1, 1.1, 2)
        if kind == 4:
            u, v = rng.choice([0.0, 1.0]), rng.uniform(0, 1)
            if rng.random() < 0.5:
                u, v = v, u
        target = (1 - u) * (1 - v) * p[0] + u * (1 - v) * p[1] + (1 - u) * v * p[2] + u * v * p[3]
        origin = target + rng.normal(size=3) * rng.choice([0.5, 3.0, 20.0])
        direction = (target - origin) * rng.choice([1.0, 0.01, 7.0]) + rng.normal(size=3) * 1e-4
        q[i, 0:12] = p.reshape(-1)
        q[i, 12:15] = origin
        q[i, 15:18] = direction
        q[i, 18] = 0.0
        q[i, 19] = np.inf if rng.random() < 0.7 else rng.uniform(0.5, 2.0)
    return q


def analytic_record(subtype, radius, z_min=-1.0, z_max=1.0, phi_max=2 * np.pi, inner_radius=0.0, height=0.0):
    a = abi.Analytic()
    a.kind, a.subtype = abi.PRIMITIVE_ANALYTIC, subtype
    a.radius, a.z_min, a.z_max, a.phi_max = radius, z_min, z_max, phi_max
    a.inner_radius, a.height = inner_radius, height
    return a


def random_analytic(rng):
    subtype = int(rng.integers(1, 4))
    r = float(rng.uniform(0.2, 3.0))
    phi = float(rng.choice([2 * np.pi, rng.uniform(0.5, 2 * np.pi)]))
    if subtype == abi.ANALYTIC_SPHERE:
        lo, hi = sorted(rng.uniform(-r, r, 2)) if rng.random() < 0.5 else (-r, r)
        if hi - lo < 1e-2 * r:
            lo, hi = -r, r
        return analytic_record(subtype, r, float(lo), float(hi), phi)
    if subtype == abi.ANALYTIC_DISK:
        return analytic_record(subtype, r, 0, 0, phi, float(rng.uniform(0, 0.8 * r) * (rng.random() < 0.5)),
                               float(rng.uniform(-1, 1)))
    lo = float(rng.uniform(-2, 0))
    return analytic_record(subtype, r, lo, lo + float(rng.uniform(0.1, 3)), phi)


def analytic_point(a, u, v):
    """The object-space point of (u, v) in double (PBRT's parameterisation)."""
    phi = u * a.phi_max
    if a.subtype == abi.ANALYTIC_DISK:
        rad = a.radius + v * (a.inner_radius - a.radius)
        return np.array([rad * np.cos(phi), rad * np.sin(phi), a.height])
    if a.subtype == abi.ANALYTIC_CYLINDER:
        return np.array([a.radius * np.cos(phi), a.radius * np.sin(phi), a.z_min + v * (a.z_max - a.z_min)])
    t0, t1 = np.arccos(np.clip(a.z_min / a.radius, -1, 1)), np.arccos(np.clip(a.z_max / a.radius, -1, 1))
    th = t0 + v * (t1 - t0)
    return a.radius * np.array([np.sin(th) * np.cos(phi), np.sin(th) * np.sin(phi), np.cos(th)])


def analytic_queries(n=20000, seed=12):
    """Spheres (whole and clipped), disks (with and without a hole) and cylinders, partial
    sweeps; rays from outside and inside aimed at points of (slightly beyond) the parameter
    square, grazing rays, and rays along the axis."""
    rng = np.random.default_rng(seed)
    q = np.zeros((n, 16), np.float32)
    for i in range(n):
        a = random_analytic(rng)
        u, v = rng.uniform(-0.05, 1.05, 2)
        target = analytic_point(a, u, v)
        if i % 7 == 0:
            origin = rng.normal(size=3) * 0.3 * a.radius  # inside
        else:
            origin = target + rng.normal(size=3) * rng.choice([0.5, 4.0, 30.0])
        direction = (target - origin) * rng.choice([1.0, 0.05, 5.0])
        if i % 11 == 0:
            direction = np.array([0.0, 0.0, rng.choice([-1.0, 1.0])])
        rec = np.frombuffer(bytes(a), np.float32)
        q[i, 0:8] = rec
        q[i, 8:11] = origin
        q[i, 11:14] = direction
        q[i, 14] = 0.0
        q[i, 15] = np.inf if rng.random() < 0.7 else rng.uniform(0.5, 2.0)
    return q
