"""CPU oracle of the reference's voxel bounce-back LBM -- TEST INFRASTRUCTURE ONLY.

Restates scripts/run_3d_window_lbm.py (voxelize :73-92, run_lbm :95-146) of
wangjianfttt/particuology_Hydraulic-penalty- in the reference's operation
order; only tests may import it.  Pinned to tests/golden/voxel_*.npz, which
make_golden.py produced by running the reference's own functions.
"""

from __future__ import annotations

import numpy as np

from .psc_oracle import C, OPP, Q, equilibrium, guo_force


def voxelize(points, center, size, radius, n):
    """Binary solid from cell centres inside spheres of one radius (:73-92)."""
    points = np.asarray(points, dtype=float).reshape(-1, 3)
    center = np.asarray(center, dtype=float)
    size = np.asarray(size, dtype=float)
    lo = center - 0.5 * size
    hi = center + 0.5 * size
    dx = size / n
    axes = [lo[k] + (np.arange(n) + 0.5) * dx[k] for k in range(3)]
    solid = np.zeros((n, n, n), dtype=bool)
    margin = radius + np.linalg.norm(dx)
    near = np.all((points >= lo - margin) & (points <= hi + margin), axis=1)
    for x, y, z in points[near]:
        b = []
        for c, k in ((x, 0), (y, 1), (z, 2)):
            b.append((max(0, int(np.floor((c - radius - lo[k]) / dx[k]))),
                      min(n - 1, int(np.ceil((c + radius - lo[k]) / dx[k])))))
        (i0, i1), (j0, j1), (k0, k1) = b
        xx = axes[0][i0:i1 + 1][:, None, None]
        yy = axes[1][j0:j1 + 1][None, :, None]
        zz = axes[2][k0:k1 + 1][None, None, :]
        solid[i0:i1 + 1, j0:j1 + 1, k0:k1 + 1] |= (xx - x) ** 2 + (yy - y) ** 2 + (zz - z) ** 2 <= radius * radius
    return solid, dx


def _moments(f, force_z):
    rho = np.sum(f, axis=0)
    ux = np.sum(f * C[:, 0, None, None, None], axis=0) / rho
    uy = np.sum(f * C[:, 1, None, None, None], axis=0) / rho
    uz = (np.sum(f * C[:, 2, None, None, None], axis=0) + 0.5 * force_z) / rho
    return rho, ux, uy, uz


def run_lbm(solid, tau, force_z, steps, return_fields=False):
    """Voxel bounce-back D3Q19 with Guo forcing (:95-146), fields as the reference returns them."""
    solid = np.asarray(solid, dtype=bool)
    shape = solid.shape
    fluid = ~solid
    f = equilibrium(np.ones(shape), np.zeros(shape), np.zeros(shape), np.zeros(shape))
    nu = (1.0 / 3.0) * (tau - 0.5)  # CS2 * (tau - 0.5), run_3d_window_lbm.py:101
    for _ in range(steps):
        rho, ux, uy, uz = _moments(f, force_z)
        ux[solid] = 0.0
        uy[solid] = 0.0
        uz[solid] = 0.0
        feq = equilibrium(rho, ux, uy, uz)
        fpost = f - (f - feq) / tau + guo_force(0.0, 0.0, force_z, ux, uy, uz, tau)
        for i in range(Q):
            f[i] = np.roll(fpost[i], shift=tuple(int(v) for v in C[i]), axis=(0, 1, 2))
        # in-place overwrite in index order, as the reference writes it (:117-119)
        for i in range(Q):
            f[i, solid] = f[OPP[i], solid].copy()
    rho, ux, uy, uz = _moments(f, force_z)
    ux[solid] = 0.0
    uy[solid] = 0.0
    uz[solid] = 0.0
    res = {
        "mean_uz_fluid": float(np.mean(uz[fluid])),
        "superficial_uz": float(np.mean(uz)),
        "max_uz": float(np.max(uz[fluid])) if np.any(fluid) else 0.0,
        "permeability_lu": nu * float(np.mean(uz)) / max(force_z, 1e-30),
        "porosity_voxel": float(np.mean(fluid)),
    }
    if return_fields:
        res.update({"ux": ux, "uy": uy, "uz": uz})
    return res
