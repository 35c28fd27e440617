"""Seeded synthetic pore windows: FCC skeleton, passive fines, preloaded fines.

The reference reads its pore windows from LIGGGHTS dumps that are not part
of its archive (scripts/run_psc_permeability_resolution.py:44-76 reads them;
README.md says the dumps are excluded).  These generators stand in for them
with the same three geometry classes and particle scales:

* ``skeleton``  -- spheres on a face-centred-cubic lattice (4 sites per cell,
  2 x 2 x 2 cells per window), radius 0.95 x the touching radius
  a / (2 sqrt 2), each centre jittered uniformly by +-2 % of the cell edge a.
* ``passive``   -- skeleton plus fines of radius 0.15 x the skeleton radius,
  placed by seeded random sequential addition in the pore space without
  overlap (periodic distances) until the solid fraction grew by 0.05.
* ``preloaded`` -- the passive fines, each moved along the line to its
  nearest skeleton sphere until it overlaps that sphere by 1-3 % of its own
  radius.

Windows are periodic for the flow, but the reference's voxeliser clips a
sphere at the box faces instead of wrapping it (psc3d.py:73-78).  So every
sphere that crosses a face is emitted again as periodic images;
``Window.owner`` maps each emitted particle back to its generating sphere.
All lengths are lattice units of a window of edge ``n``.
"""

from __future__ import annotations

from dataclasses import dataclass, field
import itertools

import numpy as np

GEOMETRY_TYPES = ("skeleton", "passive", "preloaded")


@dataclass
class Window:
    """One periodic pore window: particle table (P, 10) plus provenance."""

    n: int
    kind: str
    seed: int
    particles: np.ndarray  # (P, 10) x y z r vx vy vz wx wy wz, images included
    owner: np.ndarray  # (P,) index of the generating sphere
    is_fine: np.ndarray  # (P,) bool
    r_skeleton: float
    r_fine: float
    n_spheres: int
    meta: dict = field(default_factory=dict)

    @property
    def cells(self) -> int:
        return self.n ** 3


def fcc_skeleton(n: int, rng: np.random.Generator, cells: int = 2, radius_factor: float = 0.95,
                 jitter: float = 0.02) -> tuple[np.ndarray, float]:
    """Centres (S, 3) and radius of the jittered FCC skeleton in an n^3 box."""
    a = n / cells
    basis = np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]])
    # shift by a/4 so that no centre sits exactly on a face
    sites = np.array([(np.array(c) + b + 0.25) * a for c in itertools.product(range(cells), repeat=3) for b in basis])
    sites += rng.uniform(-jitter * a, jitter * a, size=sites.shape)
    sites %= n
    r = radius_factor * a / (2.0 * np.sqrt(2.0))
    return sites, float(r)


def _periodic_delta(d: np.ndarray, n: float) -> np.ndarray:
    return d - n * np.round(d / n)


def rsa_fines(n: int, skel: np.ndarray, r_skel: float, r_fine: float, target_volume: float,
              rng: np.random.Generator, max_trials: int = 4_000_000) -> np.ndarray:
    """Random sequential addition of fines in the pore space, no overlaps (periodic)."""
    vol_one = 4.0 / 3.0 * np.pi * r_fine ** 3
    want = int(np.ceil(target_volume / vol_one))
    placed = np.zeros((0, 3))
    batch = 4096
    trials = 0
    min_sf = (r_skel + r_fine) ** 2
    min_ff = (2.0 * r_fine) ** 2
    while len(placed) < want and trials < max_trials:
        cand = rng.uniform(0.0, n, size=(batch, 3))
        trials += batch
        d = _periodic_delta(cand[:, None, :] - skel[None, :, :], n)
        ok = np.all(np.einsum("ijk,ijk->ij", d, d) > min_sf, axis=1)
        cand = cand[ok]
        for c in cand:
            if len(placed) >= want:
                break
            if len(placed):
                d = _periodic_delta(placed - c, n)
                if np.min(np.einsum("ij,ij->i", d, d)) <= min_ff:
                    continue
            placed = np.vstack([placed, c])
    return placed


def preload(n: int, fines: np.ndarray, skel: np.ndarray, r_skel: float, r_fine: float,
            rng: np.random.Generator) -> np.ndarray:
    """Move each fine toward its nearest skeleton sphere to a 1-3 % radius overlap."""
    out = fines.copy()
    for i, c in enumerate(fines):
        d = _periodic_delta(skel - c, n)
        dist = np.sqrt(np.einsum("ij,ij->i", d, d))
        j = int(np.argmin(dist))
        overlap = rng.uniform(0.01, 0.03) * r_fine
        target = r_skel + r_fine - overlap
        direction = d[j] / max(dist[j], 1e-12)
        out[i] = (c + direction * (dist[j] - target)) % n
    return out


def periodic_images(centres: np.ndarray, radii: np.ndarray, n: int):
    """Each sphere plus its images in the 26 neighbouring boxes that reach into [0, n)^3."""
    pts, rad, own = [], [], []
    shifts = np.array(list(itertools.product((-1, 0, 1), repeat=3)), dtype=float) * n
    for i, (c, r) in enumerate(zip(centres, radii)):
        for s in shifts:
            p = c + s
            # the clipped box [floor(p - r - 1), ceil(p + r + 1)) must meet [0, n)
            if np.all(p + r + 1.0 > 0.0) and np.all(p - r - 1.0 < n):
                pts.append(p)
                rad.append(r)
                own.append(i)
    return np.asarray(pts).reshape(-1, 3), np.asarray(rad), np.asarray(own, dtype=np.int64)


def make_window(n: int, kind: str, seed: int, fines_fraction: float = 0.05, n_fines: int | None = None,
                fine_ratio: float = 0.15) -> Window:
    """One seeded window of edge n and geometry ``kind`` (see module docstring)."""
    if kind not in GEOMETRY_TYPES:
        raise ValueError(f"kind must be one of {GEOMETRY_TYPES}")
    rng = np.random.default_rng(seed)
    skel, r_skel = fcc_skeleton(n, rng)
    r_fine = fine_ratio * r_skel
    centres = [skel]
    radii = [np.full(len(skel), r_skel)]
    fine_flags = [np.zeros(len(skel), dtype=bool)]
    if kind != "skeleton":
        target = fines_fraction * n ** 3 if n_fines is None else n_fines * 4.0 / 3.0 * np.pi * r_fine ** 3
        fines = rsa_fines(n, skel, r_skel, r_fine, target, rng)
        if n_fines is not None:
            fines = fines[:n_fines]
        if kind == "preloaded":
            fines = preload(n, fines, skel, r_skel, r_fine, rng)
        centres.append(fines)
        radii.append(np.full(len(fines), r_fine))
        fine_flags.append(np.ones(len(fines), dtype=bool))
    c = np.vstack(centres)
    r = np.concatenate(radii)
    isf = np.concatenate(fine_flags)
    pts, rad, own = periodic_images(c, r, n)
    parts = np.zeros((len(pts), 10))
    parts[:, 0:3] = pts
    parts[:, 3] = rad
    return Window(n=n, kind=kind, seed=seed, particles=parts, owner=own, is_fine=isf[own], r_skeleton=r_skel,
                  r_fine=r_fine, n_spheres=len(c), meta={"n_fines": int(isf.sum())})


def batched_windows(count: int = 24, edges=(48, 64, 96, 128, 160), seed0: int = 0) -> list[Window]:
    """The uneven-window batch: edge and geometry type drawn per window from its own seed."""
    out = []
    for k in range(count):
        rng = np.random.default_rng(10_000 + seed0 + k)
        n = int(rng.choice(edges))
        kind = GEOMETRY_TYPES[int(rng.integers(0, len(GEOMETRY_TYPES)))]
        out.append(make_window(n, kind, seed0 + k))
    return out
