"""FP64 reference adjoint of the PSC-IMB permeability -- TEST INFRASTRUCTURE ONLY.

This is the NumPy discrete adjoint that the CUDA adjoint kernel is checked
against (and that is itself checked against central finite differences).
Only tests and the benchmark's checking legs import it.

Forward model (the differentiable surrogate of the reference's step):
  * smooth solid fraction: the reference counts sub-samples inside a sphere
    (src/lbm_dem/psc3d.py:79-90), which is piecewise constant in the sphere's
    centre and radius (zero derivative almost everywhere).  Here each sample
    contributes sigma((r - |x_s - X|) / eps) instead of the 0/1 indicator;
    eps -> 0 recovers the count.  Same bounding boxes and sample offsets.
  * alpha_sum = sum_p alpha_p, solid = clip(alpha_sum, 0, 1), B as psc3d.py:229.
  * static particles (u_s = 0), BGK + Noble-Torczynski + Guo, deviation
    form g = f - w (the reference's step, psc3d.py:211-232, rewritten in
    deviations; identical in exact arithmetic).
  * pull streaming; stored state S_t is post-collision; f_t = pull(S_t).
  * K = nu / (|F| N) * sum_x (1 - solid) u_F, u = (m + F/2) / rho of the
    final post-stream state (run_psc_permeability_resolution.py:144-150).
"""

from __future__ import annotations

import numpy as np

from .psc_oracle import C, OPP, Q, W, particle_bbox, particles_to_array


def sigmoid(h):
    return 0.5 * (1.0 + np.tanh(0.5 * h))


# ---------------------------------------------------------------------------
# smooth geometry
# ---------------------------------------------------------------------------
def _sample_grid(p, n, S):
    offs = (np.arange(S, dtype=np.float64) + 0.5) / S
    ix0, ix1, iy0, iy1, iz0, iz1 = particle_bbox(p[0], p[1], p[2], p[3], n)
    if ix1 <= ix0 or iy1 <= iy0 or iz1 <= iz0:
        return None
    gx = (np.arange(ix0, ix1)[:, None] + offs[None, :])  # (bx, S)
    gy = (np.arange(iy0, iy1)[:, None] + offs[None, :])
    gz = (np.arange(iz0, iz1)[:, None] + offs[None, :])
    return (ix0, ix1, iy0, iy1, iz0, iz1), gx, gy, gz


def smooth_alpha(particles, n: int, S: int, eps: float, with_grad: bool = False):
    """Per-particle smooth alpha over its clipped bbox.

    Returns list of (ids, alpha[, dalpha (4, m): d/dx, d/dy, d/dz, d/dr]).
    """
    parr = particles_to_array(particles)
    out = []
    for p in parr:
        g = _sample_grid(p, n, S)
        if g is None:
            out.append((np.zeros(0, np.int64), np.zeros(0)) + ((np.zeros((4, 0)),) if with_grad else ()))
            continue
        (ix0, ix1, iy0, iy1, iz0, iz1), gx, gy, gz = g
        dx = gx - p[0]
        dy = gy - p[1]
        dz = gz - p[2]
        # (bx, S, by, S, bz, S)
        DX = dx[:, :, None, None, None, None]
        DY = dy[None, None, :, :, None, None]
        DZ = dz[None, None, None, None, :, :]
        d = np.sqrt(DX * DX + DY * DY + DZ * DZ)
        h = (p[3] - d) / eps
        s = sigmoid(h)
        alpha = s.sum(axis=(1, 3, 5)) / S ** 3
        bx, by, bz = alpha.shape
        ii, jj, kk = np.meshgrid(np.arange(ix0, ix1), np.arange(iy0, iy1), np.arange(iz0, iz1), indexing="ij")
        ids = ((ii * n + jj) * n + kk).ravel()
        if not with_grad:
            out.append((ids, alpha.ravel()))
            continue
        ds = s * (1.0 - s) / eps / S ** 3  # d alpha / d r per sample
        dinv = np.where(d > 1e-12, 1.0 / np.maximum(d, 1e-12), 0.0)
        gr = ds.sum(axis=(1, 3, 5)).ravel()
        gxp = (ds * DX * dinv).sum(axis=(1, 3, 5)).ravel()
        gyp = (ds * DY * dinv).sum(axis=(1, 3, 5)).ravel()
        gzp = (ds * DZ * dinv).sum(axis=(1, 3, 5)).ravel()
        out.append((ids, alpha.ravel(), np.stack([gxp, gyp, gzp, gr])))
    return out


def smooth_solid(particles, n, S, eps):
    ent = smooth_alpha(particles, n, S, eps)
    asum = np.zeros(n ** 3)
    for e in ent:
        asum[e[0]] += e[1]
    return asum, np.clip(asum, 0.0, 1.0)


def bweight(solid, tau):
    return solid / (solid + tau * (1.0 - solid) + 1.0e-14)


def dbweight(solid, tau):
    D = solid + tau * (1.0 - solid) + 1.0e-14
    return (tau + 1.0e-14) / (D * D)


# ---------------------------------------------------------------------------
# deviation-form step and its vector-Jacobian product
# ---------------------------------------------------------------------------
CF = C.astype(np.float64)


def pull(S):
    out = np.empty_like(S)
    for i in range(Q):
        out[i] = np.roll(S[i], shift=tuple(int(v) for v in C[i]), axis=(0, 1, 2))
    return out


def pull_T(M):
    out = np.empty_like(M)
    for i in range(Q):
        out[i] = np.roll(M[i], shift=tuple(-int(v) for v in C[i]), axis=(0, 1, 2))
    return out


def _wq(i):
    return W[i]


def collide_dev(g, B, tau, F):
    """Post-collision deviations (static particles)."""
    F = np.asarray(F, dtype=np.float64)
    drho = g.sum(axis=0)
    rho = 1.0 + drho
    m = np.einsum("ia,i...->a...", CF, g)
    ue = (m + F[:, None, None, None]) / rho
    uu = (ue * ue).sum(axis=0)
    uF = np.einsum("a,a...->...", F, ue)
    kb = (1.0 - B) / tau
    pref = 1.0 - 0.5 / tau
    cu = np.einsum("ia,a...->i...", CF, ue)
    cF = CF @ F
    geq = W[:, None, None, None] * (drho + rho * (3.0 * cu + 4.5 * cu * cu - 1.5 * uu))
    os_ = g[OPP] - g + W[:, None, None, None] * drho - geq[OPP]
    G = pref * W[:, None, None, None] * (3.0 * (cF[:, None, None, None] - uF) + 9.0 * cu * cF[:, None, None, None])
    return g - kb * (g - geq) + B * os_ + G


def collide_dev_vjp(g, B, lam, tau, F):
    """(lambda^T dC/dg, lambda . dC/dB) at state g (per cell)."""
    F = np.asarray(F, dtype=np.float64)
    drho = g.sum(axis=0)
    rho = 1.0 + drho
    irho = 1.0 / rho
    m = np.einsum("ia,i...->a...", CF, g)
    ue = (m + F[:, None, None, None]) * irho
    uu = (ue * ue).sum(axis=0)
    kb = (1.0 - B) / tau
    pref = 1.0 - 0.5 / tau
    cu = np.einsum("ia,a...->i...", CF, ue)
    cF = CF @ F
    Wb = W[:, None, None, None]
    geq = Wb * (drho + rho * (3.0 * cu + 4.5 * cu * cu - 1.5 * uu))
    os_ = g[OPP] - g + Wb * drho - geq[OPP]
    dB = (lam * ((g - geq) / tau + os_)).sum(axis=0)
    a = kb * lam - B * lam[OPP]
    out = (1.0 - kb - B) * lam + B * lam[OPP]
    drho_bar = B * (Wb * lam).sum(axis=0) + (a * Wb * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * uu)).sum(axis=0)
    # ue_bar_a = sum_i a_i w_i rho (3 c_ia + 9 cu_i c_ia - 3 ue_a) + sum_i lam_i pref w_i (-3 F_a + 9 cF_i c_ia)
    t1 = a * Wb * rho * (3.0 + 9.0 * cu)  # coefficient of c_ia
    s1 = (a * Wb * rho * 3.0).sum(axis=0)  # coefficient of -ue_a
    t2 = lam * pref * Wb * 9.0 * cF[:, None, None, None]  # coefficient of c_ia
    s2 = (lam * pref * Wb * 3.0).sum(axis=0)  # coefficient of -F_a
    ue_bar = np.einsum("ia,i...->a...", CF, t1 + t2) - s1 * ue - s2 * F[:, None, None, None]
    m_bar = ue_bar * irho
    drho_bar = drho_bar - (ue_bar * ue).sum(axis=0) * irho
    out = out + drho_bar + np.einsum("ia,a...->i...", CF, m_bar)
    return out, dB


def moments_dev(f, F):
    F = np.asarray(F, dtype=np.float64)
    rho = 1.0 + f.sum(axis=0)
    m = np.einsum("ia,i...->a...", CF, f)
    u = (m + 0.5 * F[:, None, None, None]) / rho
    return rho, u


def permeability(S_T, solid, tau, F):
    F = np.asarray(F, dtype=np.float64)
    fmag = float(np.linalg.norm(F))
    d = F / fmag
    rho, u = moments_dev(pull(S_T), F)
    uF = np.einsum("a,a...->...", d, u)
    nu = (tau - 0.5) / 3.0
    return nu * float(((1.0 - solid) * uF).sum()) / solid.size / fmag


def forward(particles, n, S, eps, tau, F, steps, keep=False):
    asum, solid = smooth_solid(particles, n, S, eps)
    solid = solid.reshape((n, n, n))
    B = bweight(solid, tau)
    St = np.zeros((Q, n, n, n))
    states = []
    for _ in range(steps):
        if keep:
            states.append(St)
        St = collide_dev(pull(St), B, tau, F)
    return permeability(St, solid, tau, F), St, states, asum.reshape((n, n, n)), solid


def gradient(particles, n, S, eps, tau, F, steps):
    """dK/d(x, y, z, r) per particle, (P, 4), by the discrete adjoint."""
    parr = particles_to_array(particles)
    F = np.asarray(F, dtype=np.float64)
    K, S_T, states, asum, solid = forward(parr, n, S, eps, tau, F, steps, keep=True)
    B = bweight(solid, tau)
    fmag = float(np.linalg.norm(F))
    d = F / fmag
    nu = (tau - 0.5) / 3.0
    kappa = nu / (fmag * solid.size)
    fT = pull(S_T)
    rho, u = moments_dev(fT, F)
    uF = np.einsum("a,a...->...", d, u)
    cd = CF @ d
    dK_df = kappa * (1.0 - solid) * (cd[:, None, None, None] - uF) / rho
    dK_dsolid = -kappa * uF
    lam = pull_T(dK_df)
    dKdB = np.zeros_like(solid)
    for t in range(steps - 1, -1, -1):
        mu, dB = collide_dev_vjp(pull(states[t]), B, lam, tau, F)
        dKdB += dB
        lam = pull_T(mu)
    dK_dsolid = dK_dsolid + dKdB * dbweight(solid, tau)
    dK_dasum = (dK_dsolid * ((asum > 0.0) & (asum < 1.0))).ravel()
    grads = np.zeros((len(parr), 4))
    for ip, (ids, alpha, dal) in enumerate(smooth_alpha(parr, n, S, eps, with_grad=True)):
        if len(ids):
            grads[ip] = dal @ dK_dasum[ids]
    return K, grads, dKdB
