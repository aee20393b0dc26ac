"""Seeded synthetic oriented clouds standing in for the reference's public scans.

The reference benchmarks on downloaded scans (eagle, horse, bunny, torso); none are
available offline, so these generators reproduce the benchmark configurations' shapes,
sizes and density variation instead:

* ``sphere``      — points uniform by area on the unit sphere, exact normals;
* ``torus``       — uniform by area on a torus, jittered positions and perturbed normals;
* ``bumpy_sphere``— r(theta, phi) = 1 + 0.15 * sum_{l<=8} a_lm Y_lm with a_lm ~ N(0, 1/(l+1)^2),
  area-uniform candidates thinned by a smooth seeded acceptance field in [0.1, 1]
  (10x density variation), exact normals of |x| - r(theta, phi);
* ``three_tori``  — smooth union of three tori with jitter, 1% outliers, 2% flipped normals.
All return float64 numpy arrays (positions, normals) of shape (N, 3).
"""
import math

import numpy as np


def sphere(count, seed=2026):
    rng = np.random.default_rng(seed)
    n = rng.normal(size=(count, 3))
    n /= np.linalg.norm(n, axis=1)[:, None]
    return n.copy(), n


def _torus_area(rng, count, R, r):
    out_u, out_v = [], []
    total = 0
    while total < count:
        m = 2 * (count - total) + 1024
        u = rng.uniform(0, 2 * np.pi, m)
        v = rng.uniform(0, 2 * np.pi, m)
        keep = rng.uniform(size=m) < (R + r * np.cos(v)) / (R + r)
        out_u.append(u[keep])
        out_v.append(v[keep])
        total += int(keep.sum())
    u = np.concatenate(out_u)[:count]
    v = np.concatenate(out_v)[:count]
    p = np.stack([(R + r * np.cos(v)) * np.cos(u), (R + r * np.cos(v)) * np.sin(u), r * np.sin(v)], 1)
    n = np.stack([np.cos(v) * np.cos(u), np.cos(v) * np.sin(u), np.sin(v)], 1)
    return p, n


def torus(count, R=1.0, r=0.35, position_sigma=0.002, normal_sigma=0.05, seed=2026):
    rng = np.random.default_rng(seed)
    p, n = _torus_area(rng, count, R, r)
    diag = np.linalg.norm(p.max(0) - p.min(0))
    p = p + rng.normal(scale=position_sigma * diag, size=p.shape)
    n = n + rng.normal(scale=normal_sigma, size=n.shape)
    n /= np.linalg.norm(n, axis=1)[:, None]
    return p, n


class _Radius:
    """r(theta, phi) = 1 + amplitude * sum a_lm Y_lm (real, orthonormal) and its partials.

    Associated Legendre functions come from the standard upward recurrences, evaluated
    together with their theta-derivatives, so normals are exact (no finite differences).
    """

    def __init__(self, rng, lmax=8, amplitude=0.15):
        self.lmax = lmax
        self.amplitude = amplitude
        self.coef = {(l, m): rng.normal(scale=1.0 / (l + 1)) for l in range(lmax + 1) for m in range(-l, l + 1)}

    def __call__(self, theta, phi):
        x, s = np.cos(theta), np.sin(theta)
        r = np.zeros_like(theta)
        rt = np.zeros_like(theta)
        rp = np.zeros_like(theta)
        pmm = np.ones_like(theta)   # P_m^m
        dmm = np.zeros_like(theta)  # dP_m^m / dtheta
        for m in range(self.lmax + 1):
            if m > 0:
                f = -(2 * m - 1)
                pmm, dmm = f * s * pmm, f * (x * pmm + s * dmm)
            p_prev, d_prev = np.zeros_like(theta), np.zeros_like(theta)
            p_cur, d_cur = pmm, dmm
            cos_m, sin_m = np.cos(m * phi), np.sin(m * phi)
            for l in range(m, self.lmax + 1):
                if l > m:
                    p_new = ((2 * l - 1) * x * p_cur - (l + m - 1) * p_prev) / (l - m)
                    d_new = ((2 * l - 1) * (x * d_cur - s * p_cur) - (l + m - 1) * d_prev) / (l - m)
                    p_prev, d_prev, p_cur, d_cur = p_cur, d_cur, p_new, d_new
                norm = math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(l - m) / math.factorial(l + m))
                if m == 0:
                    a = self.coef[(l, 0)] * norm
                    r += a * p_cur
                    rt += a * d_cur
                else:
                    a = self.coef[(l, m)] * math.sqrt(2) * norm
                    b = self.coef[(l, -m)] * math.sqrt(2) * norm
                    trig = a * cos_m + b * sin_m
                    r += trig * p_cur
                    rt += trig * d_cur
                    rp += (b * cos_m - a * sin_m) * m * p_cur
        k = self.amplitude
        return 1.0 + k * r, k * rt, k * rp


def bumpy_sphere(count=800_000, seed=2026):
    rng = np.random.default_rng(seed)
    radius = _Radius(rng)
    # Smooth acceptance field over directions, in [0.1, 1]: low-frequency plane waves.
    waves = [(rng.normal(size=3) * 2.5, rng.uniform(0, 2 * np.pi)) for _ in range(4)]

    def acceptance(u):
        s = sum(np.sin(u @ k + ph) for k, ph in waves) / len(waves)
        return 0.1 + 0.9 * (0.5 + 0.5 * s) ** 2

    pts, nrm = [], []
    total = 0
    area_max = None
    while total < count:
        m = 6 * (count - total) + 4096
        d = rng.normal(size=(m, 3))
        d /= np.linalg.norm(d, axis=1)[:, None]
        d = d[rng.uniform(size=m) < acceptance(d)]
        theta = np.arccos(np.clip(d[:, 2], -1, 1))
        phi = np.arctan2(d[:, 1], d[:, 0])
        r, rt, rp = radius(theta, phi)
        st = np.maximum(np.sin(theta), 1e-12)
        area = r * np.sqrt(r * r + rt * rt + (rp / st) ** 2)  # surface area per unit solid angle
        if area_max is None:
            area_max = 1.5 * area.max()
        keep = rng.uniform(size=len(d)) < area / area_max
        e_t = np.stack([np.cos(theta) * np.cos(phi), np.cos(theta) * np.sin(phi), -np.sin(theta)], 1)
        e_p = np.stack([-np.sin(phi), np.cos(phi), np.zeros_like(phi)], 1)
        g = d - (rt[:, None] * e_t + (rp / st)[:, None] * e_p) / r[:, None]
        g /= np.linalg.norm(g, axis=1)[:, None]
        pts.append((r[:, None] * d)[keep])
        nrm.append(g[keep])
        total += int(keep.sum())
    return np.concatenate(pts)[:count], np.concatenate(nrm)[:count]


def three_tori(count=3_500_000, R=0.6, r=0.2, side=0.9, jitter=0.001, outliers=0.01, flipped=0.02, seed=2026):
    rng = np.random.default_rng(seed)
    centres = [np.array([side * math.cos(a), side * math.sin(a), 0.0]) / math.sqrt(3)
               for a in (np.pi / 2, np.pi / 2 + 2 * np.pi / 3, np.pi / 2 + 4 * np.pi / 3)]

    def inside(x, c):
        q = x - c
        rho = np.sqrt(q[:, 0] ** 2 + q[:, 1] ** 2)
        return (rho - R) ** 2 + q[:, 2] ** 2 < r * r

    pts, nrm = [], []
    total = 0
    while total < count:
        m = (count - total) + 4096
        k = rng.integers(0, 3, m)
        p, n = _torus_area(rng, m, R, r)
        p = p + np.stack(centres)[k]
        keep = np.ones(m, bool)
        for j, c in enumerate(centres):
            keep &= ~((k != j) & inside(p, c))
        pts.append(p[keep])
        nrm.append(n[keep])
        total += int(keep.sum())
    p = np.concatenate(pts)[:count]
    n = np.concatenate(nrm)[:count]
    diag = np.linalg.norm(p.max(0) - p.min(0))
    p = p + rng.normal(scale=jitter * diag, size=p.shape)
    lo, hi = p.min(0), p.max(0)
    o = rng.uniform(size=count) < outliers
    p[o] = rng.uniform(lo, hi, size=(int(o.sum()), 3))
    rn = rng.normal(size=(int(o.sum()), 3))
    n[o] = rn / np.linalg.norm(rn, axis=1)[:, None]
    f = rng.uniform(size=count) < flipped
    n[f] = -n[f]
    return p, n


CONFIGS = {
    1: dict(cloud=lambda: sphere(20_000), depth=6, full_depth=3, point_weight=2.0, dtype="float32",
            name="sphere 20k, depth 6, full depth 3, SPSR pw 2"),
    2: dict(cloud=lambda: torus(200_000), depth=8, full_depth=4, point_weight=4.0, dtype="float32",
            name="torus 200k (R 1, r 0.35), depth 8, full depth 4, SPSR pw 4"),
    3: dict(cloud=lambda: bumpy_sphere(800_000), depth=9, full_depth=4, point_weight=2.0, dtype="float32",
            name="bumpy sphere 800k (SH l<=8, 10x density variation), depth 9, full depth 4, SPSR pw 2"),
    4: dict(cloud=lambda: torus(100_000), depth=7, full_depth=3, point_weight=2.0, dtype="float64",
            name="torus 100k, depth 7, full depth 3, SPSR pw 2 (adjoint)"),
    5: dict(cloud=lambda: three_tori(3_500_000), depth=10, full_depth=5, point_weight=4.0, dtype="float32",
            name="three tori 3.5M with 1% outliers and 2% flipped normals, depth 10, full depth 5, SPSR pw 4"),
}
