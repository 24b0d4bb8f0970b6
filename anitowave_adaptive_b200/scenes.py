"""Seeded synthetic scenes for the FLIP-on-MSBG path (host side, numpy).

Every scene is generated once on the host and uploaded.  Randomness comes from a counter-based
splitmix64 keyed by (seed, particle slot, axis), so a scene is a pure function of its parameters
and identical on every machine.

Scenes (cell counts use the convention "a finest cell is seeded iff its centre is inside"):
  dam_break_64      64^3 unit cube, 8^3-cell blocks, 2 levels (L0 within 8 cells of the free
                    surface), column [0,0.4]x[0,0.6]x[0,1], 8 jittered particles per cell, seed 0.
  dam_drop_128      128^3, 3 levels (8/24), the same column plus a sphere r=0.12 at
                    (0.7,0.8,0.5) moving at (0,-1,0), seed 1.
  poisson_256       256^3 effective, 4 levels from the distance to 32 seeded spheres, closed box;
                    the right-hand side is the divergence of 64 seeded Gaussian velocity blobs.
  dam_drop2_256     256^3, 4 levels, column [0,0.5]x[0,0.5]x[0,1] plus two spheres r=0.1 at
                    (0.75,0.85,0.3) and (0.75,0.85,0.7) moving at (0,-2,0), seed 4, dt=1/480.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

_GOLD = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
_SEEDMUL = np.uint64(0xD1B54A32D192ED03)


def splitmix64(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = (x.astype(np.uint64) + _GOLD).astype(np.uint64)
        z = ((z ^ (z >> np.uint64(30))) * _M1).astype(np.uint64)
        z = ((z ^ (z >> np.uint64(27))) * _M2).astype(np.uint64)
        return z ^ (z >> np.uint64(31))


def uniform01(seed: int, counter: np.ndarray) -> np.ndarray:
    """24-bit uniforms in [0,1) from (seed, counter); exact in float32."""
    with np.errstate(over="ignore"):
        key = splitmix64(np.uint64(seed) * _SEEDMUL ^ np.asarray(counter, np.uint64))
    return (key >> np.uint64(40)).astype(np.float64) * (2.0 ** -24)


def normal01(seed: int, counter: np.ndarray) -> np.ndarray:
    u1 = uniform01(seed, 2 * np.asarray(counter, np.uint64))
    u2 = uniform01(seed, 2 * np.asarray(counter, np.uint64) + np.uint64(1))
    return np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2 * np.pi * u2)


@dataclass
class Scene:
    name: str
    dims: tuple
    block_size: float
    domain_min: tuple
    base_res: int
    num_levels: int
    thresholds: tuple  # level thresholds in finest cells (multiples of base_res)
    dt: float
    alpha: float = 0.95
    gravity: float = -9.81
    pos: np.ndarray = field(default=None, repr=False)  # (n,3) float32
    vel: np.ndarray = field(default=None, repr=False)  # (n,3) float32
    meta: dict = field(default_factory=dict)

    @property
    def n(self):
        return 0 if self.pos is None else self.pos.shape[0]

    @property
    def cells(self):
        return tuple(d * self.base_res for d in self.dims)


def seed_cells(N: int, inside_fn, seed: int, vel_fn=None):
    """8 stratified-jittered particles (2x2x2 sub-cells, uniform jitter) per seeded cell."""
    h = 1.0 / N
    ax = (np.arange(N) + 0.5) * h
    # iterate z-slabs to bound memory at 256^3
    pos_parts, vel_parts = [], []
    for k in range(N):
        zc = ax[k]
        yy, xx = np.meshgrid(ax, ax, indexing="ij")
        zz = np.full_like(xx, zc)
        ins = inside_fn(xx, yy, zz)
        if not ins.any():
            continue
        jj, ii = np.nonzero(ins)
        cell = (ii + N * (jj + N * k)).astype(np.uint64)
        slot = (cell[:, None] * np.uint64(8) + np.arange(8, dtype=np.uint64)[None, :]).reshape(-1)
        sub = np.arange(8)
        sx, sy, sz = (sub & 1), (sub >> 1) & 1, (sub >> 2) & 1
        base = np.stack([ii, jj, np.full_like(ii, k)], -1).astype(np.float64)
        u = np.stack([uniform01(seed, slot * np.uint64(3) + np.uint64(a)) for a in range(3)], -1)
        subo = np.stack([sx, sy, sz], -1).astype(np.float64)
        p = (np.repeat(base, 8, 0) + (np.tile(subo, (len(ii), 1)) + u) * 0.5) * h
        pos_parts.append(p.astype(np.float32))
        if vel_fn is not None:
            c = np.stack([xx[jj, ii], yy[jj, ii], zz[jj, ii]], -1)
            vel_parts.append(np.repeat(vel_fn(c), 8, 0).astype(np.float32))
    pos = np.concatenate(pos_parts, 0) if pos_parts else np.zeros((0, 3), np.float32)
    if vel_fn is None:
        vel = np.zeros_like(pos)
    else:
        vel = np.concatenate(vel_parts, 0)
    return pos, vel


def _box(lo, hi):
    return lambda x, y, z: (x > lo[0]) & (x < hi[0]) & (y > lo[1]) & (y < hi[1]) & (z > lo[2]) & (z < hi[2])


def _sphere(c, r):
    return lambda x, y, z: (x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2 < r * r


def dam_break(N=64, base_res=8, levels=2, thresholds=(8,), seed=0, dt=1.0 / 240, box=(0.4, 0.6, 1.0),
              spheres=(), name="dam_break"):
    box_fn = _box((0, 0, 0), box)

    def inside(x, y, z):
        m = box_fn(x, y, z)
        for c, r, _ in spheres:
            m = m | _sphere(c, r)(x, y, z)
        return m

    def vel_fn(c):
        v = np.zeros_like(c)
        for cc, r, vv in spheres:
            ins = ((c - np.asarray(cc)) ** 2).sum(-1) < r * r
            v[ins] = vv
        return v

    pos, vel = seed_cells(N, inside, seed, vel_fn if spheres else None)
    dims = (N // base_res,) * 3
    return Scene(name, dims, base_res / N, (0.0, 0.0, 0.0), base_res, levels, tuple(thresholds), dt,
                 pos=pos, vel=vel)


def phase_sphere(pos, center, radius) -> np.ndarray:
    """Two-phase label per particle: 1 inside the sphere (the second phase), 0 elsewhere."""
    d2 = ((np.asarray(pos, np.float64) - np.asarray(center, np.float64)) ** 2).sum(-1)
    return (d2 < radius * radius).astype(np.float32)


def config(name: str) -> Scene:
    """The named workloads (see module docstring)."""
    if name == "dam_break_64":
        return dam_break(64, 8, 2, (8,), 0, 1.0 / 240, name=name)
    if name == "dam_drop_128":
        return dam_break(128, 8, 3, (8, 24), 1, 1.0 / 240,
                         spheres=[((0.7, 0.8, 0.5), 0.12, (0.0, -1.0, 0.0))], name=name)
    if name == "dam_drop2_256":
        return dam_break(256, 8, 4, (8, 24, 56), 4, 1.0 / 480, box=(0.5, 0.5, 1.0),
                         spheres=[((0.75, 0.85, 0.3), 0.1, (0.0, -2.0, 0.0)),
                                  ((0.75, 0.85, 0.7), 0.1, (0.0, -2.0, 0.0))], name=name)
    if name.startswith("dam_break_"):  # small test variants, e.g. dam_break_16
        N = int(name.split("_")[-1])
        return dam_break(N, 8 if N >= 32 else 4, 2, (8 if N >= 32 else 4,), 0, 1.0 / 240, name=name)
    raise KeyError(name)


# ------------------------------------------------------------------------------------------------
# Poisson benchmark scene: sphere-union level map + Gaussian-blob divergence
# ------------------------------------------------------------------------------------------------
def poisson_spheres(n_spheres=32, seed=2):
    idx = np.arange(n_spheres, dtype=np.uint64)
    c = np.stack([0.1 + 0.8 * uniform01(seed, idx * np.uint64(4) + np.uint64(a)) for a in range(3)], -1)
    r = 0.03 + 0.07 * uniform01(seed, idx * np.uint64(4) + np.uint64(3))
    return c, r


def poisson_blobs(n_blobs=64, seed=3):
    idx = np.arange(n_blobs, dtype=np.uint64)
    c = np.stack([0.1 + 0.8 * uniform01(seed, idx * np.uint64(8) + np.uint64(a)) for a in range(3)], -1)
    sig = 0.02 + 0.04 * uniform01(seed, idx * np.uint64(8) + np.uint64(3))
    amp = np.stack([normal01(seed, idx * np.uint64(8) + np.uint64(4 + a)) for a in range(3)], -1)
    return c, sig, amp


def blob_velocity(X, c, sig, amp):
    """u(X) = sum_k amp_k exp(-|X-c_k|^2 / (2 sig_k^2)), X: (n,3) float64."""
    out = np.zeros_like(X)
    for k in range(c.shape[0]):
        d2 = ((X - c[k]) ** 2).sum(-1)
        g = np.exp(-d2 / (2 * sig[k] ** 2))
        out += g[:, None] * amp[k][None, :]
    return out


def sphere_surface_points(N, c, r):
    """Finest-cell 'surface' occupancy for the sphere union: centres of cells inside the union,
    returned as points (one per inside cell) so the particle level-map rule applies unchanged."""
    h = 1.0 / N
    ax = (np.arange(N) + 0.5) * h
    pts = []
    for k in range(N):
        yy, xx = np.meshgrid(ax, ax, indexing="ij")
        zz = np.full_like(xx, ax[k])
        ins = np.zeros_like(xx, dtype=bool)
        for s in range(c.shape[0]):
            ins |= (xx - c[s, 0]) ** 2 + (yy - c[s, 1]) ** 2 + (zz - c[s, 2]) ** 2 < r[s] ** 2
        jj, ii = np.nonzero(ins)
        if len(ii):
            pts.append(np.stack([xx[jj, ii], yy[jj, ii], zz[jj, ii]], -1))
    return np.concatenate(pts, 0).astype(np.float32)
