"""Seeded curve generators for the descent-step workloads.

Every random number comes from one documented PRNG so that any host (Python,
C++, a TypeScript shim) can regenerate identical bytes:

* ``splitmix64`` used counter-style: draw ``i`` of stream ``seed`` is
  ``mix(seed + (i + 1) * 0x9E3779B97F4A7C15)`` with the standard splitmix64
  finaliser (shifts 30/27/31, multipliers 0xBF58476D1CE4E5B9 and
  0x94D049BB133111EB);
* uniforms ``((z >> 11) + 0.5) * 2**-53`` in (0, 1);
* normals by Box-Muller, pairing draws ``2j`` and ``2j + 1``.

Curves are returned as ``(vertices float64[V, 3], edges int32[E, 2])``, the
``Vec3[]`` / ``Edge[]`` pair of the reference (src/core/testConfigs.ts:1-2).
``trefoil`` follows src/core/fixtures.ts:10-23.
"""
from __future__ import annotations

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, count: int) -> np.ndarray:
    """``count`` raw 64-bit draws of stream ``seed``."""
    with np.errstate(over="ignore"):
        i = np.arange(1, count + 1, dtype=np.uint64)
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + i * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def uniforms(seed: int, count: int) -> np.ndarray:
    z = splitmix64(seed, count)
    return ((z >> np.uint64(11)).astype(np.float64) + 0.5) * (2.0 ** -53)


def normals(seed: int, count: int) -> np.ndarray:
    m = (count + 1) // 2
    u = uniforms(seed, 2 * m)
    u1, u2 = u[0::2], u[1::2]
    r = np.sqrt(-2.0 * np.log(u1))
    out = np.empty(2 * m, dtype=np.float64)
    out[0::2] = r * np.cos(2.0 * np.pi * u2)
    out[1::2] = r * np.sin(2.0 * np.pi * u2)
    return out[:count]


def closed_edges(n: int, offset: int = 0) -> np.ndarray:
    i = np.arange(n, dtype=np.int32)
    return np.stack([i + offset, (i + 1) % n + offset], axis=1).astype(np.int32)


def trefoil(n: int, jitter: float = 0.0, seed: int = 0):
    """Closed trefoil (sin t + 2 sin 2t, cos t - 2 cos 2t, -sin 3t), t = 2 pi i / n,
    plus optional N(0, jitter^2) noise per coordinate."""
    t = 2.0 * np.pi * np.arange(n) / n
    v = np.stack([np.sin(t) + 2.0 * np.sin(2.0 * t), np.cos(t) - 2.0 * np.cos(2.0 * t),
                  -np.sin(3.0 * t)], axis=1)
    if jitter:
        v = v + jitter * normals(seed, 3 * n).reshape(n, 3)
    return np.ascontiguousarray(v, dtype=np.float64), closed_edges(n)


def torus_knot(n: int, p: int, q: int, jitter: float = 0.0, seed: int = 0):
    """(p, q) torus knot on the torus of radii (2, 1)."""
    t = 2.0 * np.pi * np.arange(n) / n
    r = np.cos(q * t) + 2.0
    v = np.stack([r * np.cos(p * t), r * np.sin(p * t), -np.sin(q * t)], axis=1)
    if jitter:
        v = v + jitter * normals(seed, 3 * n).reshape(n, 3)
    return np.ascontiguousarray(v, dtype=np.float64), closed_edges(n)


def _polygon_length(v: np.ndarray) -> float:
    return float(np.linalg.norm(np.roll(v, -1, axis=0) - v, axis=1).sum())


def random_walk_knot(n: int, seed: int = 1, total_length: float = 10.0):
    """Closed random-walk polygon: n 3-D Gaussian steps of sigma = 1/sqrt(n) from the
    origin, closed by removing the linear drift (i/n)(x_n - x_0), rescaled so the
    closed polygon has the given total length."""
    steps = normals(seed, 3 * n).reshape(n, 3) / np.sqrt(n)
    walk = np.concatenate([np.zeros((1, 3)), np.cumsum(steps, axis=0)], axis=0)
    drift = walk[n] - walk[0]
    v = walk[:n] - (np.arange(n)[:, None] / n) * drift[None, :]
    v = v * (total_length / _polygon_length(v))
    return np.ascontiguousarray(v, dtype=np.float64), closed_edges(n)


def loop_network(loops: int = 12, n: int = 1024, junctions: int = 8, seed: int = 5,
                 spacing: float = 4.0):
    """``loops`` random-walk loops of n vertices (total length 10 each) on a
    square grid of the given spacing, joined by junctions//2 bridge edges whose
    endpoints become degree-3 (Y) junction vertices."""
    side = int(np.ceil(np.sqrt(loops)))
    verts, edges = [], []
    for l in range(loops):
        v, e = random_walk_knot(n, seed=seed * 1000 + l)
        v = v - v.mean(axis=0) + np.array([(l % side) * spacing, (l // side) * spacing, 0.0])
        verts.append(v)
        edges.append(e + l * n)
    u = uniforms(seed * 7919 + 17, 4 * junctions)
    bridges = []
    used = set()
    for j in range(junctions // 2):
        a = int(u[4 * j] * loops) % loops
        b = (a + 1 + int(u[4 * j + 1] * (loops - 1))) % loops
        va = a * n + int(u[4 * j + 2] * n) % n
        vb = b * n + int(u[4 * j + 3] * n) % n
        while va in used:
            va = a * n + (va - a * n + 1) % n
        while vb in used:
            vb = b * n + (vb - b * n + 1) % n
        used.update((va, vb))
        bridges.append((va, vb))
    V = np.concatenate(verts, axis=0)
    Ed = np.concatenate(edges + [np.asarray(bridges, dtype=np.int32).reshape(-1, 2)], axis=0)
    return np.ascontiguousarray(V), np.ascontiguousarray(Ed.astype(np.int32))


def seeded_pins(n_vertices: int, count: int, seed: int = 11) -> np.ndarray:
    """``count`` distinct vertex indices."""
    u = uniforms(seed, 4 * count)
    out: list[int] = []
    for x in u:
        v = int(x * n_vertices) % n_vertices
        if v not in out:
            out.append(v)
        if len(out) == count:
            break
    return np.asarray(out, dtype=np.int32)


def batch_curves(count: int = 64, vmin: int = 256, vmax: int = 4096, seed: int = 3):
    """Uneven batch: sizes log-uniform in [vmin, vmax]; shapes cycle through
    trefoil, torus knots (2,3)/(3,5)/(2,7) and random walks, 1/3 each."""
    u = uniforms(seed, 2 * count)
    curves = []
    torus = [(2, 3), (3, 5), (2, 7)]
    for c in range(count):
        n = int(round(np.exp(np.log(vmin) + u[c] * (np.log(vmax) - np.log(vmin)))))
        kind = c % 3
        if kind == 0:
            v, e = trefoil(n, jitter=0.01, seed=seed * 100 + c)
        elif kind == 1:
            p, q = torus[int(u[count + c] * 3) % 3]
            v, e = torus_knot(n, p, q, jitter=0.01, seed=seed * 100 + c)
        else:
            v, e = random_walk_knot(n, seed=seed * 100 + c)
        curves.append((v, e))
    return curves
