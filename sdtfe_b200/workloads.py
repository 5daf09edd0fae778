"""Seeded synthetic particle sets and map settings of the benchmark workloads.

No external data is read; every generator is a pure function of its seed
(numpy ``default_rng``).  Positions are returned as the reference's (N, 4)
float64 rows (column 3 zero), already rounded to float32 where the workload
says the positions are float32.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class MapSpec:
    grid_dim: int
    n_samples: int
    box_len: float
    box_len_z: float
    center: tuple
    delta_sample: float = 0.0

    @property
    def rays(self) -> int:
        return self.grid_dim * self.grid_dim * self.n_samples


def _rows(xyz: np.ndarray, f32: bool) -> np.ndarray:
    pos = np.zeros((len(xyz), 4), np.float64)
    pos[:, :3] = xyz.astype(np.float32) if f32 else xyz
    return pos


def _isotropic(rng, n):
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    return d


def clusters_r2(rng, n_points: int, n_clusters: int, r_max: float, centres: np.ndarray) -> np.ndarray:
    """Points in isotropic clusters with density ~ r^-2 truncated at r_max:
    enclosed mass grows linearly in r, so r = r_max * U."""
    counts = np.full(n_clusters, n_points // n_clusters)
    counts[: n_points - counts.sum()] += 1
    owner = np.repeat(np.arange(n_clusters), counts)
    r = r_max * rng.random(n_points)
    return centres[owner] + r[:, None] * _isotropic(rng, n_points)


def uniform_box(n=32768, seed=1):
    """Plain method, CPU-runnable: N uniform float64 in [0,1]^3, 256^2 map,
    4 samples per pixel, the full unit box projected along z."""
    rng = np.random.default_rng(seed)
    pos = _rows(rng.random((n, 3)), f32=False)
    return pos, MapSpec(256, 4, 1.0, 1.0, (0.5, 0.5, 0.5))


def clustered_box(n=1 << 20, seed=2, n_clusters=100, r_max=0.02, grid_dim=2048, n_samples=16):
    """Clustered single map: half uniform in [0,1]^3, half in n_clusters r^-2
    clusters (truncation r_max) with uniform centres, wrapped periodically into
    [0,1); float32 positions; 2048^2 z-projection with 16 samples per pixel."""
    rng = np.random.default_rng(seed)
    n_u = n // 2
    u = rng.random((n_u, 3))
    c = clusters_r2(rng, n - n_u, n_clusters, r_max, rng.random((n_clusters, 3)))
    xyz = np.concatenate([u, c]) % 1.0
    return _rows(xyz, f32=True), MapSpec(grid_dim, n_samples, 1.0, 1.0, (0.5, 0.5, 0.5))


def halo_cutout(n, seed, bg_frac=0.2, r_max=1.0):
    """One halo cutout: an r^-2 cluster of radius r_max at the origin plus a
    uniform background in [-1,1]^3; float32 positions."""
    rng = np.random.default_rng(seed)
    n_bg = int(round(bg_frac * n))
    bg = rng.uniform(-1.0, 1.0, size=(n_bg, 3))
    cl = clusters_r2(rng, n - n_bg, 1, r_max, np.zeros((1, 3)))
    return _rows(np.concatenate([cl, bg]), f32=True)


def cutout_specs(n_cutouts=64, n_min=10_000, n_max=500_000, seed=3, sides=(256, 512, 1024),
                 n_samples=8):
    """Batched cutouts: (particle count, cutout seed, map) per cutout; counts
    log-uniform in [n_min, n_max], map side drawn uniformly from `sides`, box
    2 x 2 x 2 about the origin.  The particles are halo_cutout(n, seed)."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(n_min), np.log(n_max), n_cutouts)).astype(int)
    out = []
    for i, n in enumerate(ns):
        side = int(rng.choice(sides))
        out.append((int(n), seed * 1000 + i, MapSpec(side, n_samples, 2.0, 2.0, (0.0, 0.0, 0.0))))
    return out


def cutout_batch(**kw):
    """cutout_specs with the particles generated: [(pos4, MapSpec)]."""
    return [(halo_cutout(n, s), spec) for n, s, spec in cutout_specs(**kw)]


def perturbed_lattice(n_side=192, sigma_frac=0.3, extra_frac=0.3, n_clusters=2000, r_max=0.01,
                      seed=5):
    """Large field: n_side^3 lattice in [0,1)^3 with Gaussian displacements of
    sigma_frac * spacing, plus extra_frac * n_side^3 points in r^-2 clusters;
    float32 positions, wrapped into [0,1)."""
    rng = np.random.default_rng(seed)
    h = 1.0 / n_side
    g = (np.arange(n_side) + 0.5) * h
    lat = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    lat = lat + rng.normal(scale=sigma_frac * h, size=lat.shape)
    n_extra = int(round(extra_frac * len(lat)))
    c = clusters_r2(rng, n_extra, n_clusters, r_max, rng.random((n_clusters, 3)))
    return _rows(np.concatenate([lat, c]) % 1.0, f32=True)


@dataclass
class Request:
    t: float          # arrival time, seconds from the start of the stream
    cutout: int
    axis: int
    spec: MapSpec


def serving_stream(n_cutouts=256, n_min=10_000, n_max=2_000_000, n_requests=512, rate=100.0,
                   seed=4, sides=(128, 256, 512, 1024, 2048), s_min=4, s_max=16):
    """Serving stream: particle counts of the resident cutouts (log-uniform in
    [n_min, n_max]) and a Poisson arrival trace at `rate` requests/s; each
    request draws a cutout, a projection axis (z, x, y), a map side from
    `sides` and s_min..s_max samples per pixel.  Cutouts are built like the
    clustered single map, clustered_box(n, seed * 1000 + i); maps cover the
    unit box."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(n_min), np.log(n_max), n_cutouts)).astype(int)
    t = np.cumsum(rng.exponential(1.0 / rate, n_requests))
    reqs = []
    for k in range(n_requests):
        spec = MapSpec(int(rng.choice(sides)), int(rng.integers(s_min, s_max + 1)), 1.0, 1.0,
                       (0.5, 0.5, 0.5))
        reqs.append(Request(float(t[k]), int(rng.integers(n_cutouts)), int(rng.integers(3)), spec))
    return ns, reqs


def serving_cutouts(n_distinct=32, n_min=10_000, n_max=500_000, seed=4):
    """Particle counts (log-uniform in [n_min, n_max]) and seeds of the
    distinct cutout triangulations behind the serving stream's handles;
    handle i holds its own device copy of cutout i % n_distinct."""
    rng = np.random.default_rng(seed + 17)
    ns = np.exp(rng.uniform(np.log(n_min), np.log(n_max), n_distinct)).astype(int)
    return [(int(n), seed * 1000 + i) for i, n in enumerate(ns)]
