"""GPU drop-in for the reference's voxel bounce-back window LBM.

``voxelize`` and ``run_lbm`` keep the names, arguments and results of
scripts/run_3d_window_lbm.py (:73-92, :95-146) -- the drag-proxy solver the
older coupled loop uses -- and run in libpscb200.so (psc_voxelize_spheres,
psc_bounceback_step) in exact FP64, bit-identical to the reference.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _native as nat
from .engine import require_cuda, stream_handle, vp

Q = 19


def voxelize(points, center, size, radius: float, n: int, device=None):
    """(solid bool (n, n, n), dx (3,)): cells whose centre lies inside a sphere of ``radius``."""
    dev = require_cuda(device)
    points = np.asarray(points, dtype=np.float64).reshape(-1, 3)
    center = np.asarray(center, dtype=np.float64)
    size = np.asarray(size, dtype=np.float64)
    lo = center - 0.5 * size
    hi = center + 0.5 * size
    dx = size / n
    # the reference keeps only spheres within radius + |dx| of the box (:79-80)
    margin = radius + np.linalg.norm(dx)
    near = points[np.all((points >= lo - margin) & (points <= hi + margin), axis=1)]
    with torch.cuda.device(dev):
        solid = torch.zeros(n ** 3, dtype=torch.uint8, device=dev)
        pts = torch.from_numpy(np.ascontiguousarray(near)).to(dev)
        lo_c = (ctypes.c_double * 3)(*lo)
        dx_c = (ctypes.c_double * 3)(*dx)
        nat.call("psc_voxelize_spheres", vp(pts), int(len(near)), lo_c, dx_c, float(radius), n, n, n, vp(solid),
                 stream_handle(dev))
        out = solid.cpu().numpy().reshape(n, n, n).astype(bool)
    return out, dx


def run_lbm(solid, tau: float, force_z: float, steps: int, return_fields: bool = False, device=None) -> dict:
    """Voxel bounce-back D3Q19 with Guo forcing along z; same result dict as the reference."""
    dev = require_cuda(device)
    solid_np = np.asarray(solid, dtype=bool)
    nx, ny, nz = solid_np.shape
    N = nx * ny * nz
    with torch.cuda.device(dev):
        s = torch.from_numpy(np.ascontiguousarray(solid_np.astype(np.uint8)).reshape(-1)).to(dev)
        f = [torch.empty(Q * N, dtype=torch.float64, device=dev) for _ in range(2)]
        mom = torch.empty(4 * N, dtype=torch.float64, device=dev)
        st = stream_handle(dev)
        nat.call("psc_init_equilibrium", nat.STORE_F64_EXACT, 1.0, vp(f[0]), N, st)
        cur = 0
        for _ in range(int(steps)):
            nat.call("psc_bounceback_step", vp(f[cur]), vp(f[1 - cur]), vp(s), nx, ny, nz, float(tau), 0.0, 0.0,
                     float(force_z), nat.STEP_COLLIDE, None, st)
            cur = 1 - cur
        nat.call("psc_bounceback_step", vp(f[cur]), None, vp(s), nx, ny, nz, float(tau), 0.0, 0.0, float(force_z),
                 nat.STEP_MOMENTS, vp(mom), st)
        m = mom.view(4, nx, ny, nz).cpu().numpy()
    ux, uy, uz = m[1], m[2], m[3]
    fluid = ~solid_np
    nu = (1.0 / 3.0) * (tau - 0.5)  # CS2 * (tau - 0.5), run_3d_window_lbm.py:101
    res = {
        "mean_uz_fluid": float(np.mean(uz[fluid])),
        "superficial_uz": float(np.mean(uz)),
        "max_uz": float(np.max(uz[fluid])) if np.any(fluid) else 0.0,
        "permeability_lu": nu * float(np.mean(uz)) / max(force_z, 1e-30),
        "porosity_voxel": float(np.mean(fluid)),
        "speed_slice": uz[:, :, nz // 2].copy(),
        "solid_slice": solid_np[:, :, nz // 2].copy(),
    }
    if return_fields:
        res.update({"ux": ux.copy(), "uy": uy.copy(), "uz": uz.copy()})
    return res
