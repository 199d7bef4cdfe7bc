"""Seeded synthetic initial conditions for the gravity-step workloads.

The reference spawns its galaxies from ``std::random_device`` seeds
(GalaxyEngine/src/Particles/particlesSpawning.cpp:134-136), which is not
reproducible, so the workloads here are generated from explicit seeds:

* ``disk2d``      exponential disk, scale length 1.0 truncated at 5.0, uniform
                  angle, masses 1/N each plus a central point mass of 0.1,
                  circular velocities from the enclosed mass plus Gaussian
                  dispersion 0.02 per component (N=16,384 disk workload).
* ``two_disks2d`` two such disks, centres 10.0 apart on the x axis, relative
                  speed 0.5 on an offset (parabolic-style) approach
                  (N=1,048,576 two-disk workload).
* ``plummer3d``   Plummer sphere, scale radius 1.0, positions by inverse-CDF
                  sampling, velocities by the Aarseth-Henon-Wielen (1974)
                  rejection method, masses 1/N (N=4,194,304 workload).
* ``batch_sizes`` particle counts log-uniform in [lo, hi] (batched workload).

Every generator returns a dict of contiguous float32 arrays ``x, y, (z,)
vx, vy, (vz,) m`` plus ``id`` (uint32, 0..N-1).
"""
from __future__ import annotations

import math

import numpy as np


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def _enclosed_disk_mass(r, mdisk, h=1.0, rmax=5.0):
    """Mass of a truncated exponential disk inside radius r."""
    norm = 1.0 - math.exp(-rmax / h) * (1.0 + rmax / h)
    return mdisk * (1.0 - np.exp(-r / h) * (1.0 + r / h)) / norm


def _disk_particles(rng, n_disk, m_part, m_center, G=1.0, h=1.0, rmax=5.0, sigma=0.02):
    u = rng.random(n_disk)
    r = -h * np.log(1.0 - u * (1.0 - math.exp(-rmax / h)))
    phi = rng.random(n_disk) * 2.0 * math.pi
    x, y = r * np.cos(phi), r * np.sin(phi)
    menc = _enclosed_disk_mass(r, n_disk * m_part, h, rmax) + m_center
    vc = np.sqrt(G * menc / np.maximum(r, 1e-12))
    vx = -vc * np.sin(phi) + rng.normal(0.0, sigma, n_disk)
    vy = vc * np.cos(phi) + rng.normal(0.0, sigma, n_disk)
    return x, y, vx, vy


def _pack(x, y, vx, vy, m, z=None, vz=None):
    out = dict(x=np.ascontiguousarray(x, np.float32), y=np.ascontiguousarray(y, np.float32),
               vx=np.ascontiguousarray(vx, np.float32), vy=np.ascontiguousarray(vy, np.float32),
               m=np.ascontiguousarray(m, np.float32))
    if z is not None:
        out["z"] = np.ascontiguousarray(z, np.float32)
        out["vz"] = np.ascontiguousarray(vz, np.float32)
    out["id"] = np.arange(len(x), dtype=np.uint32)
    return out


def disk2d(n=16384, seed=0, G=1.0, m_center=0.1, total_n=None, center=(0.0, 0.0),
           bulk_v=(0.0, 0.0), rng=None):
    """One exponential disk of n particles: n-1 disk particles of mass
    1/total_n (total_n defaults to n) plus one central point mass."""
    rng = _rng(seed) if rng is None else rng
    total_n = n if total_n is None else total_n
    mp = 1.0 / total_n
    x, y, vx, vy = _disk_particles(rng, n - 1, mp, m_center, G)
    x = np.concatenate([[0.0], x]) + center[0]
    y = np.concatenate([[0.0], y]) + center[1]
    vx = np.concatenate([[0.0], vx]) + bulk_v[0]
    vy = np.concatenate([[0.0], vy]) + bulk_v[1]
    m = np.full(n, mp)
    m[0] = m_center
    return _pack(x, y, vx, vy, m)


def two_disks2d(n=1048576, seed=0, G=1.0, separation=10.0, rel_speed=0.5, angle_deg=30.0):
    """Two disks of n/2 particles each, centres (-sep/2, 0) and (+sep/2, 0),
    bulk velocities +/-(v cos a, -v sin a) with v = rel_speed/2."""
    rng = _rng(seed)
    half = n // 2
    v = 0.5 * rel_speed
    a = math.radians(angle_deg)
    d1 = disk2d(half, G=G, total_n=n, center=(-0.5 * separation, 0.0),
                bulk_v=(v * math.cos(a), -v * math.sin(a)), rng=rng)
    d2 = disk2d(n - half, G=G, total_n=n, center=(0.5 * separation, 0.0),
                bulk_v=(-v * math.cos(a), v * math.sin(a)), rng=rng)
    out = {k: np.concatenate([d1[k], d2[k]]) for k in ("x", "y", "vx", "vy", "m")}
    return _pack(out["x"], out["y"], out["vx"], out["vy"], out["m"])


def plummer3d(n=4194304, seed=0, a=1.0, G=1.0, m_frac_max=0.999):
    """Plummer sphere (total mass 1).  Radii by inverse CDF of the cumulative
    mass fraction u in [0, m_frac_max) (the outermost 0.1% is not sampled, a
    common truncation that keeps radii finite); speeds by the rejection
    sampling of q^2 (1-q^2)^(7/2) (Aarseth, Henon & Wielen 1974)."""
    rng = _rng(seed)
    u = rng.random(n) * m_frac_max
    r = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)

    def iso(k):
        ct = 2.0 * rng.random(k) - 1.0
        st = np.sqrt(1.0 - ct * ct)
        ph = 2.0 * math.pi * rng.random(k)
        return st * np.cos(ph), st * np.sin(ph), ct

    ux, uy, uz = iso(n)
    q = np.empty(n)
    todo = np.arange(n)
    while len(todo):
        xq = rng.random(len(todo))
        yq = 0.1 * rng.random(len(todo))
        ok = yq < xq * xq * (1.0 - xq * xq) ** 3.5
        q[todo[ok]] = xq[ok]
        todo = todo[~ok]
    vesc = np.sqrt(2.0 * G / a) * (1.0 + (r / a) ** 2) ** -0.25
    speed = q * vesc
    wx, wy, wz = iso(n)
    m = np.full(n, 1.0 / n)
    return _pack(r * ux, r * uy, speed * wx, speed * wy, m, z=r * uz, vz=speed * wz)


def batch_sizes(count=512, lo=1024, hi=262144, seed=2):
    """Particle counts log-uniform in [lo, hi]."""
    rng = _rng(seed)
    return np.exp(rng.uniform(math.log(lo), math.log(hi), count)).astype(np.int64)
