"""CPU oracle for the D3Q19 PSC-IMB step -- TEST INFRASTRUCTURE ONLY.

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` may import it.  The product path (the
``particuology_hydraulic_penalty_b200`` package) runs on the CUDA extension
and fails loudly when it is missing.

What it restates
----------------
The reference kernel ``src/lbm_dem/psc3d.py`` of
wangjianfttt/particuology_Hydraulic-penalty- (pure NumPy).  Every function
below cites the reference lines it follows.  The arithmetic is written in the
reference's operation order (same associativity, same divisions by ``CS2``,
no fused multiply-add, sequential population sums) so that the oracle is
bit-identical to the reference on the same inputs; the loops themselves are
restructured (vectorised sub-sample voxelisation, per-particle sparse lists
for both the dense and the sparse solver, in-place buffers).

Pinning
-------
``tests/golden/make_golden.py`` imports the reference itself and stores its
outputs as ``tests/golden/*.npz``; ``tests/test_oracle_golden.py`` requires
this oracle to reproduce them bit-exactly (fields) and to round-off
(force / torque sums, whose NumPy pairwise order differs between the dense
and sparse reference classes).

Extension beyond the reference (flagged where used): a general body-force
vector ``F = (fx, fy, fz)``.  For ``F = (0, 0, fz)`` every expression reduces
exactly to the reference's ``body_force_z`` form.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

# ---------------------------------------------------------------------------
# D3Q19 tables, same index order as psc3d.py:17-43.
# ---------------------------------------------------------------------------
C = np.array(
    [
        [0, 0, 0],
        [1, 0, 0], [-1, 0, 0],
        [0, 1, 0], [0, -1, 0],
        [0, 0, 1], [0, 0, -1],
        [1, 1, 0], [-1, -1, 0],
        [1, -1, 0], [-1, 1, 0],
        [1, 0, 1], [-1, 0, -1],
        [1, 0, -1], [-1, 0, 1],
        [0, 1, 1], [0, -1, -1],
        [0, 1, -1], [0, -1, 1],
    ],
    dtype=np.int64,
)
W = np.array([1.0 / 3.0] + [1.0 / 18.0] * 6 + [1.0 / 36.0] * 12, dtype=np.float64)
OPP = np.array([0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17], dtype=np.int64)
CS2 = 1.0 / 3.0
Q = 19

PARTICLE_FIELDS = ("x", "y", "z", "r", "vx", "vy", "vz", "wx", "wy", "wz")


def particles_to_array(particles) -> np.ndarray:
    """(P, 10) float64 array [x, y, z, r, vx, vy, vz, wx, wy, wz].

    Accepts an array already in that layout or objects with those attributes
    (the reference's ``Particle3D``, psc3d.py:46-57).
    """
    if isinstance(particles, np.ndarray):
        arr = np.asarray(particles, dtype=np.float64)
        if arr.ndim != 2 or arr.shape[1] != 10:
            raise ValueError("particle array must have shape (P, 10)")
        return arr
    rows = [[float(getattr(p, k)) for k in PARTICLE_FIELDS] for p in particles]
    return np.asarray(rows, dtype=np.float64).reshape(len(rows), 10)


# ---------------------------------------------------------------------------
# Geometry: sub-sampled solid fraction.
# ---------------------------------------------------------------------------
def particle_bbox(x: float, y: float, z: float, r: float, n: int) -> tuple[int, int, int, int, int, int]:
    """Clipped bounding box [lo, hi) per axis, psc3d.py:73-78 / 156-161."""
    ix0 = max(0, int(np.floor(x - r - 1.0)))
    ix1 = min(n, int(np.ceil(x + r + 1.0)))
    iy0 = max(0, int(np.floor(y - r - 1.0)))
    iy1 = min(n, int(np.ceil(y + r + 1.0)))
    iz0 = max(0, int(np.floor(z - r - 1.0)))
    iz1 = min(n, int(np.ceil(z + r + 1.0)))
    return ix0, ix1, iy0, iy1, iz0, iz1


def particle_counts(x: float, y: float, z: float, r: float, n: int, subsamples: int):
    """Inside-sample counts of one sphere over its clipped bbox.

    Follows psc3d.py:68-94 (and the dense copy :153-173): offsets
    ``(k + 0.5) / S``, per-axis ``dx = (i + o) - x`` and the test
    ``(dx*dx + dy*dy) + dz*dz <= r*r`` in float64.  Returns the flat node ids
    (ascending, i.e. the reference's ix/iy/iz loop order) and integer counts of
    the cells with a non-zero count.
    """
    s = max(1, int(subsamples))
    offs = (np.arange(s, dtype=np.float64) + 0.5) / s
    ix0, ix1, iy0, iy1, iz0, iz1 = particle_bbox(x, y, z, r, n)
    if ix1 <= ix0 or iy1 <= iy0 or iz1 <= iz0:
        return np.zeros(0, dtype=np.int64), np.zeros(0, dtype=np.int64)
    rr = r * r
    dx = (np.arange(ix0, ix1, dtype=np.int64)[:, None] + offs[None, :]) - x
    dy = (np.arange(iy0, iy1, dtype=np.int64)[:, None] + offs[None, :]) - y
    dz = (np.arange(iz0, iz1, dtype=np.int64)[:, None] + offs[None, :]) - z
    dx2, dy2, dz2 = dx * dx, dy * dy, dz * dz
    nyb, nzb = iy1 - iy0, iz1 - iz0
    counts = np.empty((ix1 - ix0, nyb, nzb), dtype=np.int64)
    # (dx2 + dy2) + dz2 for one ix slab at a time: shape (S, nyb, S, nzb, S)
    for a in range(ix1 - ix0):
        dxy = dx2[a][:, None, None] + dy2[None, :, :]  # (S, nyb, S)
        d2 = dxy[:, :, :, None, None] + dz2[None, None, None, :, :]  # (S, nyb, S, nzb, S)
        counts[a] = (d2 <= rr).sum(axis=(0, 2, 4))
    ii, jj, kk = np.nonzero(counts)
    ids = ((ii + ix0) * n + (jj + iy0)) * n + (kk + iz0)
    return ids.astype(np.int64), counts[ii, jj, kk]


@dataclass
class Geometry:
    """Sparse geometry: per-particle ascending node ids and alphas."""

    n: int
    subsamples: int
    node_ids: list
    counts: list
    alpha_vals: list
    alpha_sum_flat: np.ndarray
    solid: np.ndarray


def voxelize(particles, n: int, subsamples: int) -> Geometry:
    """Solid fraction and per-particle node lists.

    psc3d.py:328-345 (sparse) and :151-179 (dense).  ``alpha = count / S^3``
    (:90 / :173); the per-cell sum runs over particles in index order starting
    from 0.0, which is what both ``np.add.at`` per particle (:339-341) and the
    dense ``alpha_p.sum(axis=0)`` (:174) compute; ``solid = clip(sum, 0, 1)``.
    """
    parr = particles_to_array(particles)
    s = max(1, int(subsamples))
    n3 = n * n * n
    alpha_sum = np.zeros(n3, dtype=np.float64)
    ids_l, cnt_l, val_l = [], [], []
    denom = float(s ** 3)
    for p in parr:
        ids, cnt = particle_counts(p[0], p[1], p[2], p[3], n, s)
        vals = cnt / denom
        if len(ids):
            alpha_sum[ids] += vals  # ids are unique within one particle
        ids_l.append(ids)
        cnt_l.append(cnt)
        val_l.append(vals)
    solid = np.clip(alpha_sum.reshape((n, n, n)), 0.0, 1.0)
    return Geometry(n, s, ids_l, cnt_l, val_l, alpha_sum, solid)


def dense_alpha(geo: Geometry) -> np.ndarray:
    """Dense (P, n, n, n) alpha field of the dense reference class (psc3d.py:141,173)."""
    n = geo.n
    out = np.zeros((len(geo.node_ids), n * n * n), dtype=np.float64)
    for ip, (ids, vals) in enumerate(zip(geo.node_ids, geo.alpha_vals)):
        out[ip, ids] = vals
    return out.reshape((len(geo.node_ids), n, n, n))


def _node_xyz(ids: np.ndarray, n: int):
    ix = ids // (n * n)
    rem = ids - ix * n * n
    iy = rem // n
    iz = rem - iy * n
    return ix, iy, iz


def solid_velocity(particles, geo: Geometry):
    """alpha-weighted rigid-body velocity, psc3d.py:347-373 (dense :181-206).

    ``r = (i + 0.5) - X`` without periodic wrap; ``v = V + w x r`` in the
    reference's term order; contributions summed in particle order from 0.0,
    then divided by the alpha sum where it exceeds 1e-14.
    """
    parr = particles_to_array(particles)
    n = geo.n
    n3 = n * n * n
    us = np.zeros((3, n3), dtype=np.float64)
    for p, ids, alpha in zip(parr, geo.node_ids, geo.alpha_vals):
        if len(ids) == 0:
            continue
        ix, iy, iz = _node_xyz(ids, n)
        rx = ix + 0.5 - p[0]
        ry = iy + 0.5 - p[1]
        rz = iz + 0.5 - p[2]
        vx = p[4] + p[8] * rz - p[9] * ry
        vy = p[5] + p[9] * rx - p[7] * rz
        vz = p[6] + p[7] * ry - p[8] * rx
        us[0, ids] += alpha * vx
        us[1, ids] += alpha * vy
        us[2, ids] += alpha * vz
    mask = geo.alpha_sum_flat > 1.0e-14
    us[:, mask] /= geo.alpha_sum_flat[mask]
    return us.reshape((3, n, n, n))


# ---------------------------------------------------------------------------
# Collision pieces.
# ---------------------------------------------------------------------------
def equilibrium(rho, ux, uy, uz) -> np.ndarray:
    """Second-order D3Q19 equilibrium, psc3d.py:97-103 (same operation order)."""
    uu = ux * ux + uy * uy + uz * uz
    out = np.empty((Q, *np.shape(rho)), dtype=np.float64)
    for i in range(Q):
        cx, cy, cz = C[i]
        cu = cx * ux + cy * uy + cz * uz
        out[i] = W[i] * rho * (1.0 + cu / CS2 + 0.5 * cu * cu / (CS2 * CS2) - 0.5 * uu / CS2)
    return out


def guo_force(fx, fy, fz, ux, uy, uz, tau) -> np.ndarray:
    """Guo forcing term, psc3d.py:106-114 (same operation order)."""
    out = np.empty((Q, *np.shape(ux)), dtype=np.float64)
    pref = 1.0 - 0.5 / tau
    uf = ux * fx + uy * fy + uz * fz
    for i in range(Q):
        cx, cy, cz = C[i]
        cu = cx * ux + cy * uy + cz * uz
        cf = cx * fx + cy * fy + cz * fz
        out[i] = pref * W[i] * ((cf - uf) / CS2 + cu * cf / (CS2 * CS2))
    return out


def moments(f: np.ndarray, force=(0.0, 0.0, 0.0)):
    """rho and the half-force-shifted velocity, psc3d.py:211-214 / 243-246.

    Sums run sequentially over the population axis (NumPy ``axis=0``).  With
    ``force = (0, 0, fz)`` this is exactly ``ux = mx / rho``,
    ``uz = (mz + 0.5 fz) / rho``; other components are the flagged extension.
    """
    fx, fy, fz = (float(v) for v in force)
    rho = np.sum(f, axis=0)
    ux = (np.sum(f * C[:, 0, None, None, None], axis=0) + 0.5 * fx) / rho
    uy = (np.sum(f * C[:, 1, None, None, None], axis=0) + 0.5 * fy) / rho
    uz = (np.sum(f * C[:, 2, None, None, None], axis=0) + 0.5 * fz) / rho
    return rho, ux, uy, uz


def collide(f: np.ndarray, solid: np.ndarray, us, tau: float, force=(0.0, 0.0, 0.0)):
    """Noble-Torczynski PSC collision + Guo forcing, psc3d.py:211-236.

    Returns the post-collision populations and the node IMB momentum
    ``(imb_mx, imb_my, imb_mz)``.  Reproduces the reference's quirks: the
    second half-force shift ``u_eff = u + F/(2 rho)`` (:217-219), forcing added
    unweighted by ``1 - B`` (:230-232), the ``+1e-14`` in ``B`` (:229).
    """
    fx, fy, fz = (float(v) for v in force)
    rho, ux, uy, uz = moments(f, force)
    ux_e = ux + 0.5 * fx / rho
    uy_e = uy + 0.5 * fy / rho
    uz_e = uz + 0.5 * fz / rho
    feq_f = equilibrium(rho, ux_e, uy_e, uz_e)
    omega_bgk = -(f - feq_f) / tau
    if us is None:
        zero = np.zeros_like(rho)
        feq_s = equilibrium(rho, zero, zero, zero)
    else:
        feq_s = equilibrium(rho, us[0], us[1], us[2])
    omega_s = f[OPP] - f + feq_s - feq_f[OPP]
    alpha = np.clip(solid, 0.0, 1.0)
    b = alpha / (alpha + tau * (1.0 - alpha) + 1.0e-14)
    post = f + ((1.0 - b) * omega_bgk + b * omega_s + guo_force(fx, fy, fz, ux_e, uy_e, uz_e, tau))
    bo = b * omega_s
    imb = np.stack([np.sum(bo * C[:, k, None, None, None], axis=0) for k in range(3)])
    return post, imb


def stream_push(f: np.ndarray) -> np.ndarray:
    """Fully periodic push streaming ``np.roll(f_i, c_i)``, psc3d.py:239-242."""
    out = np.empty_like(f)
    for i in range(Q):
        out[i] = np.roll(f[i], shift=tuple(int(v) for v in C[i]), axis=(0, 1, 2))
    return out


def inlet_correction(i: int, inlet_rho: float, inlet_u) -> float:
    """Moving-wall bounce-back term 2 w_i rho_in (c_i . u_in) / cs^2 of the velocity inlet."""
    cx, cy, cz = (int(v) for v in C[i])
    cu = cx * np.float64(inlet_u[0]) + cy * np.float64(inlet_u[1]) + cz * np.float64(inlet_u[2])
    return 2.0 * (W[i] * np.float64(inlet_rho)) * cu / CS2


def stream_push_open_x(f: np.ndarray, inlet_rho: float, inlet_u) -> np.ndarray:
    """Push streaming open along x (an extension: the reference is periodic in
    every direction, psc3d.py:239-242).  Velocity inlet at x = 0 by moving-wall
    bounce-back (Ladd 1994): a population entering from outside (c_x = +1) is
    the node's own post-collision population of the opposite direction plus
    2 w_i rho_in (c_i . u_in) / cs^2, which injects exactly rho_in u_in per unit
    face area.  Zero-gradient outflow at x = nx - 1: a population entering from
    outside (c_x = -1) is the post-collision value of the plane x = nx - 1
    itself, shifted in y and z like any other.  y and z stay periodic."""
    out = stream_push(f)
    for i in range(Q):
        cx, cy, cz = (int(v) for v in C[i])
        if cx == 1:
            out[i, 0] = f[OPP[i], 0] + inlet_correction(i, inlet_rho, inlet_u)
        elif cx == -1:
            out[i, -1] = np.roll(f[i, -1], shift=(cy, cz), axis=(0, 1))
    return out


def unstream_pull(f: np.ndarray) -> np.ndarray:
    """Inverse of :func:`stream_push`."""
    out = np.empty_like(f)
    for i in range(Q):
        out[i] = np.roll(f[i], shift=tuple(-int(v) for v in C[i]), axis=(0, 1, 2))
    return out


def particle_loads(particles, geo: Geometry, imb: np.ndarray):
    """Per-particle IMB force and torque, psc3d.py:375-407 (sparse form).

    ``owner = alpha / max(alpha_sum, 1e-14)``, ``F_node = -owner * imb``,
    torque arms ``r = (i + 0.5) - X`` without wrap.  The dense reference
    (:255-281) sums the same node terms over the full lattice, which differs
    only in NumPy's pairwise summation order.
    """
    parr = particles_to_array(particles)
    n = geo.n
    imx, imy, imz = (imb[k].ravel() for k in range(3))
    P = len(parr)
    forces = np.zeros((P, 3), dtype=np.float64)
    torques = np.zeros((P, 3), dtype=np.float64)
    total = np.zeros(3, dtype=np.float64)
    for ip, (p, ids, alpha) in enumerate(zip(parr, geo.node_ids, geo.alpha_vals)):
        if len(ids) == 0:
            continue
        owner = alpha / np.maximum(geo.alpha_sum_flat[ids], 1.0e-14)
        nfx = -owner * imx[ids]
        nfy = -owner * imy[ids]
        nfz = -owner * imz[ids]
        ix, iy, iz = _node_xyz(ids, n)
        rx = ix + 0.5 - p[0]
        ry = iy + 0.5 - p[1]
        rz = iz + 0.5 - p[2]
        forces[ip] = [float(nfx.sum()), float(nfy.sum()), float(nfz.sum())]
        torques[ip] = [
            float((ry * nfz - rz * nfy).sum()),
            float((rz * nfx - rx * nfz).sum()),
            float((rx * nfy - ry * nfx).sum()),
        ]
        total += forces[ip]
    fluid = np.array([imb[0].sum(), imb[1].sum(), imb[2].sum()])
    residual = float(np.linalg.norm(total + fluid))
    return forces, torques, residual


def has_motion(particles) -> bool:
    parr = particles_to_array(particles)
    return bool(len(parr)) and bool(np.any(parr[:, 4:10] != 0.0))


# ---------------------------------------------------------------------------
# Whole solver (mirrors the reference classes' state and diagnostics).
# ---------------------------------------------------------------------------
class OracleSolver:
    """CPU restatement of ``PscD3Q19`` / ``SparsePscD3Q19`` (psc3d.py:117-407).

    ``force`` generalises ``body_force_z``; pass ``body_force_z`` for the
    reference form.  The dense and sparse reference classes share the
    collision and differ only in summation order of the load sums, so one
    class serves both.
    """

    def __init__(self, n, particles, tau=0.72, subsamples=4, body_force_z=0.0,
                 static_geometry=False, force=None, inlet=None):
        self.n = int(n)
        # inlet = (rho_in, (ux, uy, uz)): open along x (stream_push_open_x), an
        # extension beyond the reference; None: periodic, the reference.  An
        # open window starts from the rest equilibrium taken as the
        # post-collision state and streamed with its open boundaries (for a
        # periodic window that is the equilibrium itself).
        self.inlet = inlet
        self.particles = particles
        self.tau = float(tau)
        self.subsamples = int(subsamples)
        self.force = (0.0, 0.0, float(body_force_z)) if force is None else tuple(float(v) for v in force)
        self.static_geometry = bool(static_geometry)
        self.geo: Geometry | None = None
        shape = (self.n,) * 3
        self.rho = np.ones(shape)
        self.ux = np.zeros(shape)
        self.uy = np.zeros(shape)
        self.uz = np.zeros(shape)
        self.f = equilibrium(self.rho, self.ux, self.uy, self.uz)
        if self.inlet is not None:
            self.f = stream_push_open_x(self.f, *self.inlet)
        self.solid = np.zeros(shape)
        self.imb = np.zeros((3, *shape))
        P = len(particles_to_array(particles))
        self.hydro_forces = np.zeros((P, 3))
        self.hydro_torques = np.zeros((P, 3))
        self.momentum_residual = 0.0

    def rebuild_geometry(self):
        self.geo = voxelize(self.particles, self.n, self.subsamples)
        self.solid = self.geo.solid

    def collide_stream_psc(self) -> dict:
        """One step, psc3d.py:208-253."""
        if (not self.static_geometry) or self.geo is None:
            self.rebuild_geometry()
        us = solid_velocity(self.particles, self.geo) if has_motion(self.particles) else None
        post, self.imb = collide(self.f, self.solid, us, self.tau, self.force)
        self.hydro_forces, self.hydro_torques, self.momentum_residual = particle_loads(
            self.particles, self.geo, self.imb)
        self.f = stream_push(post) if self.inlet is None else stream_push_open_x(post, *self.inlet)
        self.rho, self.ux, self.uy, self.uz = moments(self.f, self.force)
        hf, ht = self.hydro_forces, self.hydro_torques
        return {
            "solid_volume_lu": float(np.sum(self.solid)),
            "mean_uz": float(np.mean(self.uz)),
            "momentum_residual": float(self.momentum_residual),
            "max_force": float(np.max(np.linalg.norm(hf, axis=1))) if len(hf) else 0.0,
            "max_torque": float(np.max(np.linalg.norm(ht, axis=1))) if len(ht) else 0.0,
        }


def darcy_permeability(solid: np.ndarray, u_along: np.ndarray, tau: float, force_mag: float) -> dict:
    """Darcy K from the final state, run_psc_permeability_resolution.py:144-150."""
    fluid_weight = 1.0 - solid
    n3 = solid.size
    fluid_volume = float(np.sum(fluid_weight))
    weighted = u_along * fluid_weight
    superficial = float(np.sum(weighted) / n3)
    nu = (tau - 0.5) / 3.0
    return {
        "porosity_psc": fluid_volume / n3,
        "superficial_u": superficial,
        "mean_u_fluid": float(np.sum(weighted) / max(fluid_volume, 1.0e-300)),
        "permeability_lu": float(nu * superficial / max(force_mag, 1.0e-300)),
    }


def collide_trt_deviation(g: np.ndarray, solid: np.ndarray, tau: float, tau_minus: float, force=(0.0, 0.0, 0.0)):
    """Two-relaxation-time variant of :func:`collide` (static particles), on deviations g = f - w.

    EXTENSION beyond the reference (which is BGK only, psc3d.py:221): the
    fluid operator relaxes the symmetric part (f_i + f_opp)/2 with 1/tau and
    the antisymmetric part (f_i - f_opp)/2 with 1/tau_minus; Guo's
    antisymmetric term 3 w c.F takes the prefactor 1 - 1/(2 tau_minus).  The
    PSC term and B are the reference's.  tau_minus = tau is BGK.
    """
    F = np.asarray(force, dtype=np.float64)
    Cf = C.astype(np.float64)
    Wb = W[:, None, None, None]
    drho = g.sum(axis=0)
    rho = 1.0 + drho
    m = np.einsum("ia,i...->a...", Cf, g)
    ue = (m + F[:, None, None, None]) / rho
    uu = (ue * ue).sum(axis=0)
    uF = np.einsum("a,a...->...", F, ue)
    cu = np.einsum("ia,a...->i...", Cf, ue)
    cF = (Cf @ F)[:, None, None, None]
    geq = Wb * (drho + rho * (3.0 * cu + 4.5 * cu * cu - 1.5 * uu))
    alpha = np.clip(solid, 0.0, 1.0)
    B = alpha / (alpha + tau * (1.0 - alpha) + 1.0e-14)
    os_ = g[OPP] - g + Wb * drho - geq[OPP]
    gp, gm = 0.5 * (g + g[OPP]), 0.5 * (g - g[OPP])
    ep, em = 0.5 * (geq + geq[OPP]), 0.5 * (geq - geq[OPP])
    fluid = -(gp - ep) / tau - (gm - em) / tau_minus
    pref_p, pref_m = 1.0 - 0.5 / tau, 1.0 - 0.5 / tau_minus
    G = Wb * (pref_p * (-3.0 * uF + 9.0 * cu * cF) + pref_m * 3.0 * cF)
    return g + (1.0 - B) * fluid + B * os_ + G
