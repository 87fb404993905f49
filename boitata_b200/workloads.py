"""Five seeded synthetic kriging workloads, c1 to c5 (described below).

No public dataset is named for this path, so every input is generated here
with the reference tests' 64-bit LCG (crates/estimation/src/kernel.rs:132-137:
state = state * 6364136223846793005 + 1442695040888963407, u = (state >> 11)
/ 2^53, one step before each draw) and its Box-Muller normals
(batch.rs:639-642). Draws are taken in the order documented per workload, so
another implementation can regenerate the same inputs.

  c1  2,000 samples uniform in 1000 x 1000 x 200 m, lognormal values
      (log-sd 1); spherical (nugget 0.1, sill 0.9, 150 m, ratios 1 and 1/3);
      50 x 50 x 20 grid of 20 x 20 x 10 m blocks; Search(ranges=(300, 300,
      100), max_samples=16).
  c2  400 vertical drill holes (collars on a 25 m grid, +-1 m jitter), 125
      composites at 2 m: 50,000 samples; lognormal values (log-sd 1.2), 5 %
      zeros; nugget 0.05 + spherical 0.5 (80 m) + exponential 0.45 (250 m),
      rotation (30, 10, 0), ratios (0.75, 0.25) - one anisotropy shared by
      the structures, as the reference's Variogram holds; 200 x 200 x 80
      grid of 2.5 x 2.5 x 3.125 m blocks (3.2M); Search(radius=250,
      octant=True, max_per_sector=4, max_samples=32).
  c3  c1's box with a sample density rising 10x along x (2,000 samples);
      Search(radius=150, min_samples=4, max_samples=64); simple kriging with
      mean 1.0 on every 10th target.
  c4  20,000 samples in c1's box, Gaussian-field values; leave-one-out
      loss and gradient (see c4 below).
"""

from dataclasses import dataclass

import numpy as np

from .geometry import Geometry
from .search import Search
from .variogram import Structure, Variogram

A = np.uint64(6364136223846793005)
C = np.uint64(1442695040888963407)


def lcg(seed, n):
    """The first n uniforms of the LCG from `seed` (states s_1..s_n), vectorised by doubling."""
    if n <= 0:
        return np.empty(0)
    with np.errstate(over="ignore"):
        states = np.array([np.uint64(seed) * A + C], dtype=np.uint64)
        a, c = A, C  # map s -> a s + c advances by len(states)
        while len(states) < n:
            k = len(states)
            states = np.concatenate([states, states * a + c])
            a, c = a * a, a * c + c
            assert len(states) == 2 * k
    return (states[:n] >> np.uint64(11)).astype(np.float64) / float(1 << 53)


class Stream:
    """Sequential draws from the LCG (uniform and Box-Muller normal)."""

    def __init__(self, seed, capacity=1 << 16):
        self.seed, self.pos = seed, 0
        self._buf = lcg(seed, capacity)

    def uniform(self, n):
        need = self.pos + n
        if need > len(self._buf):
            self._buf = lcg(self.seed, max(need, 2 * len(self._buf)))
        out = self._buf[self.pos:need]
        self.pos = need
        return out.copy()

    def normal(self, n):
        uv = self.uniform(2 * n).reshape(n, 2)
        u = np.maximum(uv[:, 0], 1e-300)
        return np.sqrt(-2.0 * np.log(u)) * np.cos(2.0 * np.pi * uv[:, 1])


@dataclass
class Workload:
    name: str
    coords: np.ndarray
    values: np.ndarray
    variogram: Variogram
    search: Search
    geometry: Geometry
    kind: str = "ordinary"
    mean: float = 0.0


def c1(seed=1):
    s = Stream(seed)
    xyz = s.uniform(3 * 2000).reshape(2000, 3) * np.array([1000.0, 1000.0, 200.0])
    values = np.exp(s.normal(2000))
    vg = Variogram([Structure("spherical", 0.9, 150.0)], nugget=0.1, ratios=(1.0, 1.0 / 3.0))
    search = Search(ranges=(300.0, 300.0, 100.0), max_samples=16, min_samples=1)
    geo = Geometry((0.0, 0.0, 0.0), (20.0, 20.0, 10.0), (50, 50, 20))
    return Workload("c1", xyz, values, vg, search, geo)


def c2(seed=2, holes=20):
    s = Stream(seed)
    i, j = np.meshgrid(np.arange(holes), np.arange(holes), indexing="xy")
    jitter = s.uniform(2 * holes * holes).reshape(holes * holes, 2) * 2.0 - 1.0
    cx = 12.5 + 25.0 * i.ravel() + jitter[:, 0]
    cy = 12.5 + 25.0 * j.ravel() + jitter[:, 1]
    z = 249.0 - 2.0 * np.arange(125)
    xyz = np.column_stack([np.repeat(cx, 125), np.repeat(cy, 125), np.tile(z, holes * holes)])
    n = len(xyz)
    values = np.exp(1.2 * s.normal(n))
    values[s.uniform(n) < 0.05] = 0.0
    vg = Variogram([Structure("spherical", 0.5, 80.0), Structure("exponential", 0.45, 250.0)], nugget=0.05,
                   rotation=(30.0, 10.0, 0.0), ratios=(0.75, 0.25))
    search = Search(radius=250.0, octant=True, max_per_sector=4, max_samples=32)
    geo = Geometry((0.0, 0.0, 0.0), (2.5, 2.5, 3.125), (200, 200, 80))
    return Workload("c2", xyz, values, vg, search, geo)


def c3(seed=3):
    s = Stream(seed)
    u = s.uniform(3 * 2000).reshape(2000, 3)
    x = (-1.0 + np.sqrt(1.0 + 99.0 * u[:, 0])) / 0.009  # density proportional to 1 + 9 x / 1000 on [0, 1000]
    xyz = np.column_stack([x, 1000.0 * u[:, 1], 200.0 * u[:, 2]])
    values = np.exp(s.normal(2000))
    vg = Variogram([Structure("spherical", 0.9, 150.0)], nugget=0.1, ratios=(1.0, 1.0 / 3.0))
    search = Search(radius=150.0, min_samples=4, max_samples=64)
    geo = Geometry((0.0, 0.0, 0.0), (20.0, 20.0, 10.0), (50, 50, 20))
    return Workload("c3", xyz, values, vg, search, geo, kind="mixed-sk", mean=1.0)


WORKLOADS = {"c1": c1, "c2": c2, "c3": c3}


def gaussian_field(xyz, normals, rng=150.0, device=None):
    """Values of a zero-mean Gaussian field with covariance exp(-3 h / rng) (sill 1) at xyz: L @ normals
    for the Cholesky factor L of the covariance matrix (batch.rs:626-648 makes its test fields this way).
    With `device` (a torch device) the FP64 matrix and its factor are formed there."""
    if device is None:
        d = xyz[:, None, :] - xyz[None, :, :]
        cov = np.exp(-3.0 * np.sqrt((d * d).sum(-1)) / rng)
        return np.linalg.cholesky(cov) @ normals
    import torch

    x = torch.as_tensor(xyz, dtype=torch.float64, device=device)
    cov = torch.cdist(x, x)
    cov.mul_(-3.0 / rng).exp_()
    low = torch.linalg.cholesky(cov)
    del cov
    out = low @ torch.as_tensor(normals, dtype=torch.float64, device=device)
    return out.cpu().numpy()


def c4(n=20000, seed=4, device=None):
    """Leave-one-out gradient workload: n samples in c1's box with Gaussian-field values (exponential
    covariance, sill 1, range 150 m); kriging variogram nugget 0.05 + spherical 0.5 (100 m) + exponential
    0.45 (250 m), rotation (30, 10, 0), ratios (0.75, 0.5): 10 parameters; each held-out sample kriged from
    its 32 nearest samples (Search(radius=inf, max_samples=32)), neighbourhoods frozen at these values."""
    s = Stream(seed)
    xyz = s.uniform(3 * n).reshape(n, 3) * np.array([1000.0, 1000.0, 200.0])
    values = gaussian_field(xyz, s.normal(n), device=device)
    vg = Variogram([Structure("spherical", 0.5, 100.0), Structure("exponential", 0.45, 250.0)], nugget=0.05,
                   rotation=(30.0, 10.0, 0.0), ratios=(0.75, 0.5))
    search = Search(radius=float("inf"), max_samples=32, min_samples=1)
    return Workload("c4", xyz, values, vg, search, None)


WORKLOADS["c4"] = c4


def c5(holes=1600, seed=5):
    """Large and ill-conditioned: holes (1600 -> 200,000 composites) in 40 clusters in a 1000 x 1000 x 250 m
    box, 125 composites at 2 m each, plus a copy of 10 % of the samples 0.01 m away (beyond the 1e-6 m
    coincident guard); lognormal values; Gaussian variogram (nugget 1e-4, sill 1, range 200 m), near-singular
    systems; 400 x 400 x 64 blocks (10.24M); octant search, 8 per octant, 64 at most, radius 300 m."""
    s = Stream(seed)
    centres = s.uniform(2 * 40).reshape(40, 2) * 1000.0
    u = s.uniform(3 * holes).reshape(holes, 3)
    c = centres[(u[:, 0] * 40).astype(int) % 40]
    cx = np.clip(c[:, 0] + (u[:, 1] - 0.5) * 100.0, 0.0, 1000.0)
    cy = np.clip(c[:, 1] + (u[:, 2] - 0.5) * 100.0, 0.0, 1000.0)
    z = 249.0 - 2.0 * np.arange(125)
    xyz = np.column_stack([np.repeat(cx, 125), np.repeat(cy, 125), np.tile(z, holes)])
    n = len(xyz)
    pick = np.nonzero(s.uniform(n) < 0.1)[0]
    twins = xyz[pick] + np.array([0.01, 0.0, 0.0])
    xyz = np.vstack([xyz, twins])
    values = np.exp(s.normal(len(xyz)))
    vg = Variogram([Structure("gaussian", 1.0, 200.0)], nugget=1e-4)
    search = Search(radius=300.0, octant=True, max_per_sector=8, max_samples=64)
    geo = Geometry((0.0, 0.0, 0.0), (2.5, 2.5, 250.0 / 64), (400, 400, 64))
    return Workload("c5", xyz, values, vg, search, geo)


WORKLOADS["c5"] = c5
