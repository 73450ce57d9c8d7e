"""Seeded synthetic systems for the energy/force path.

Stand-ins for the benchmark inputs (no dataset is shipped or downloaded):

* :func:`water_box` - periodic cubic water box: O on an ``n^3`` lattice with
  +-0.2 A uniform jitter, two H per O at 0.9572 A and 104.52 deg with a
  uniformly random orientation.  64 waters in 12.42 A, 4096 in 49.7 A and
  32768 in 99.4 A are the 192 / 12,288 / 98,304-atom boxes.
* :func:`organic_molecule` / :func:`molecule_batch` - random-walk bonded chains
  with species drawn H .50, C .30, N .07, O .08, S .02, F .02, Cl .01, steps
  U(1.1, 1.6) A and a 0.9 A minimum pair distance.
* :func:`request_stream` - a Poisson stream of single-point and MD requests
  with log-uniform atom counts.

Coordinates are float64 in Angstrom, species are atomic numbers.
"""

from __future__ import annotations

import dataclasses
from typing import List, Optional

import numpy as np

WATER_OH = 0.9572
WATER_HOH_DEG = 104.52
WATER_SPACING = 12.42 / 4.0  # A between lattice O (about 1 g/cm^3)


def _random_rotations(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniform random rotation matrices from normalised Gaussian quaternions."""
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], axis=1)


@dataclasses.dataclass
class System:
    """One system: coordinates [n,3] (A), atomic numbers [n], optional 3x3 cell
    (rows are lattice vectors, FeNNol's ``cells[b]`` convention)."""

    coordinates: np.ndarray
    species: np.ndarray
    cell: Optional[np.ndarray] = None

    @property
    def natoms(self) -> int:
        return int(self.species.shape[0])


def water_box(n_side: int, box: Optional[float] = None, seed: int = 0,
              jitter: float = 0.2) -> System:
    """Cubic periodic box of ``n_side^3`` waters (O, H, H per molecule)."""
    if box is None:
        box = WATER_SPACING * n_side
    rng = np.random.default_rng(seed)
    a = box / n_side
    g = (np.arange(n_side) + 0.5) * a
    ox, oy, oz = np.meshgrid(g, g, g, indexing="ij")
    o = np.stack([ox.ravel(), oy.ravel(), oz.ravel()], -1)
    o = o + rng.uniform(-jitter, jitter, size=o.shape)
    nmol = o.shape[0]
    half = np.deg2rad(WATER_HOH_DEG) / 2
    local = np.array([[np.sin(half), 0.0, np.cos(half)],
                      [-np.sin(half), 0.0, np.cos(half)]]) * WATER_OH
    rot = _random_rotations(rng, nmol)
    h = o[:, None, :] + np.einsum("mij,kj->mki", rot, local)
    xyz = np.concatenate([o[:, None, :], h], axis=1).reshape(-1, 3)
    species = np.tile(np.array([8, 1, 1], dtype=np.int32), nmol)
    return System(xyz, species, np.eye(3) * box)


SPECIES_DRAW = (1, 6, 7, 8, 16, 9, 17)
SPECIES_PROB = (0.50, 0.30, 0.07, 0.08, 0.02, 0.02, 0.01)


def organic_molecule(n: int, rng: np.random.Generator, step=(1.1, 1.6),
                     min_dist: float = 0.9, max_tries: int = 200) -> System:
    """Random-walk chain of ``n`` atoms, every pair at least ``min_dist`` apart."""
    species = rng.choice(np.array(SPECIES_DRAW, dtype=np.int32), size=n,
                         p=np.array(SPECIES_PROB))
    while True:
        xyz = np.zeros((n, 3))
        ok = True
        for k in range(1, n):
            for _ in range(max_tries):
                d = rng.standard_normal(3)
                d /= np.linalg.norm(d)
                cand = xyz[k - 1] + d * rng.uniform(*step)
                if np.min(np.linalg.norm(xyz[:k] - cand, axis=1)) >= min_dist:
                    xyz[k] = cand
                    break
            else:
                ok = False
                break
        if ok:
            return System(xyz - xyz.mean(0), species.astype(np.int32), None)


def molecule_batch(n_mol: int, seed: int = 0, nmin: int = 10, nmax: int = 40) -> List[System]:
    rng = np.random.default_rng(seed)
    return [organic_molecule(int(rng.integers(nmin, nmax + 1)), rng) for _ in range(n_mol)]


def water_cluster_box(natoms_target: int, seed: int) -> System:
    """Periodic water box with about ``natoms_target`` atoms (k^3 waters)."""
    k = max(2, int(round((natoms_target / 3) ** (1 / 3))))
    return water_box(k, seed=seed)


@dataclasses.dataclass
class Request:
    arrival_s: float
    system: System
    kind: str  # "ef" (single point energy+forces) or "md" (MD continuation)
    md_steps: int = 0


def request_stream(n_requests: int, rate_hz: float = 2000.0, seed: int = 0,
                   nmin: int = 8, nmax: int = 5000, md_fraction: float = 0.3,
                   md_steps: int = 100, pool_size: Optional[int] = None) -> List[Request]:
    """Poisson arrivals; atom counts log-uniform in [nmin, nmax]; half chains,
    half periodic water boxes; ``md_fraction`` of requests are MD continuations.

    With ``pool_size`` the systems are drawn from that many pre-generated ones
    (sizes log-uniform as above) instead of one new system per request, which
    keeps generating long streams fast."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_hz, size=n_requests))

    def new_system() -> System:
        n = int(round(np.exp(rng.uniform(np.log(nmin), np.log(nmax)))))
        if rng.uniform() < 0.5 or n < 24:
            return organic_molecule(n, rng)
        return water_cluster_box(n, seed=int(rng.integers(1 << 30)))

    pool = [new_system() for _ in range(pool_size)] if pool_size else None
    out = []
    for k in range(n_requests):
        sys_ = pool[int(rng.integers(len(pool)))] if pool else new_system()
        kind = "md" if rng.uniform() < md_fraction else "ef"
        out.append(Request(float(t[k]), sys_, kind, md_steps if kind == "md" else 0))
    return out
