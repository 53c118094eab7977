"""Synthetic workloads on the sphere (host side, numpy): velocity fields,
initial tracers and their exact solutions.

Deformational vortex flow: the vortex roll-up of the reference
(VortexRollup::solve, src/pdes/hyperbolic/vortex_rollup.cpp:31-63, and its
exact solution tests/experiments/vortex_rollup_on_sphere/exact_rollup.h:25-50:
rho = rho0 cos(theta'), V_t = (3 sqrt 3 / 2) sech^2(rho) tanh(rho),
omega = V_t / rho) turning about an axis p instead of the z axis.  Every point
rotates about p with angular speed omega(theta'), theta' the latitude relative
to p, so the velocity is V(x) = omega (p x x), and the exact solution of
h_t + V . grad h = 0 for any initial field h0 is h0 rotated back about p by
omega t.  With a tilted axis both the longitude and latitude derivatives
(LAMBDA and THETA) are needed, as in the cosine bell.
"""
import numpy as np


def unit(v):
    v = np.asarray(v, dtype=np.float64)
    return v / np.linalg.norm(v)


def seeded_axis(seed):
    rng = np.random.default_rng(seed)
    return unit(rng.standard_normal(3))


def east_north(xyz):
    x, y, z = xyz.T
    lam = np.arctan2(y, x)
    th = np.arctan2(z, np.sqrt(x * x + y * y))
    e_lam = np.stack([-np.sin(lam), np.cos(lam), np.zeros_like(lam)], axis=1)
    e_th = np.stack([-np.sin(th) * np.cos(lam), -np.sin(th) * np.sin(lam), np.cos(th)], axis=1)
    return e_lam, e_th


def vortex_omega(xyz, axis, rho0=3.0):
    s = np.clip(xyz @ axis, -1.0, 1.0)
    rho = rho0 * np.sqrt(1.0 - s * s)
    vt = 1.5 * np.sqrt(3.0) * (1.0 / np.cosh(rho)) ** 2 * np.tanh(rho)
    with np.errstate(divide="ignore", invalid="ignore"):
        om = np.where(np.abs(rho) < 4 * np.finfo(float).eps, 0.0, vt / rho)
    return om


def vortex_coefficients(xyz, axis, rho0=3.0):
    """Per-node (cu, cv): east and north velocity components (sphere radius 1),
    for f = -(cu D_lambda h + cv D_theta h)."""
    V = vortex_omega(xyz, axis, rho0)[:, None] * np.cross(axis[None, :], xyz)
    e_lam, e_th = east_north(xyz)
    return (V * e_lam).sum(1), (V * e_th).sum(1)


def rotate_about(xyz, axis, angle):
    """Rodrigues rotation of each point about `axis` by its own angle."""
    c, s = np.cos(angle)[:, None], np.sin(angle)[:, None]
    k = axis[None, :]
    return xyz * c + np.cross(k, xyz) * s + k * (xyz @ axis)[:, None] * (1 - c)


def tracer_set(T, seed):
    """T tracers: alternately cosine bells (radius 0.35) and Gaussian hills, seeded centres."""
    rng = np.random.default_rng(seed)
    cen = rng.standard_normal((T, 3))
    cen /= np.linalg.norm(cen, axis=1)[:, None]
    kinds = np.arange(T) % 2
    widths = np.where(kinds == 0, 0.35, rng.uniform(4.0, 10.0, T))
    return cen, kinds, widths


def tracer_field(xyz, cen, kinds, widths):
    out = np.zeros((xyz.shape[0], len(cen)))
    for t in range(len(cen)):
        if kinds[t] == 0:
            r = np.arccos(np.clip(xyz @ cen[t], -1.0, 1.0))
            R = widths[t]
            out[:, t] = np.where(r < R, 0.5 * (1 + np.cos(np.pi * r / R)), 0.0)
        else:
            out[:, t] = np.exp(-widths[t] * ((xyz - cen[t]) ** 2).sum(1))
    return out


def vortex_exact(xyz, axis, tracers, t, rho0=3.0):
    back = rotate_about(xyz, axis, -vortex_omega(xyz, axis, rho0) * t)
    return tracer_field(back, *tracers)
