"""Helpers the DEM coupling drivers wrap around the solver.

The reference's synchronised PSC-IMB <-> DEM driver (coupling_sync/
couple_psc_liggghts.py) converts LIGGGHTS state to lattice units, advances
the solver to a quasi-steady state or by a fixed step count every macro
step, and converts the loads back to SI.  LIGGGHTS itself (an external
shared library) stays outside this package; these functions take plain
arrays so any DEM code can drive the GPU solver the same way.

* ``apply_si_scaling``        run_local_lbm_liggghts_coupled.py:68-98
* ``psc_particles_from_state`` run_local_lbm_liggghts_coupled.py:159-177
* ``lbm_converge``            couple_psc_liggghts.py:284-296
* ``lbm_transient_advance``   couple_psc_liggghts.py:299-310
"""

from __future__ import annotations

import math

import numpy as np

CS2 = 1.0 / 3.0
BOX_SIZE = 0.009
R_HELIUM = 2077.1


def apply_si_scaling(resolution: int, tau: float, temperature_k: float = 773.15, pressure_pa: float = 2.0e5,
                     mu_he: float = 3.7e-5, box_size: float = BOX_SIZE) -> dict:
    """Lattice <-> SI scales for helium at (T, p) (run_local_lbm_liggghts_coupled.py:68-98).

    nu_lu = cs^2 (tau - 1/2); dx = box / resolution; dt = nu_lu dx^2 / nu_phys;
    force scale rho dx^4 / dt^2, torque scale force scale x dx.
    """
    rho_he = pressure_pa / (R_HELIUM * temperature_k)
    nu_phys = mu_he / rho_he
    nu_lu = CS2 * (tau - 0.5)
    dx = box_size / resolution
    dt = nu_lu * dx * dx / nu_phys
    u_scale = dx / dt
    force_scale = rho_he * dx ** 4 / (dt * dt)
    return {
        "rho_he_kg_m3": rho_he, "nu_phys_m2_s": nu_phys, "nu_lu": nu_lu, "dx_m": dx, "dt_s": dt,
        "u_scale_m_s": u_scale, "force_scale_N_per_lu": force_scale,
        "torque_scale_Nm_per_lu": force_scale * dx,
        "velocity_lu_per_m_s": 1.0 / u_scale, "angular_lu_per_rad_s": dt,
    }


def psc_particles_from_state(x, v, omega, radius, resolution: int, velocity_lu_scale: float,
                             angular_lu_scale: float, box_size: float = BOX_SIZE) -> np.ndarray:
    """(P, 10) lattice-unit particle table from SI positions, velocities, spins and radii
    (run_local_lbm_liggghts_coupled.py:159-177)."""
    x = np.asarray(x, dtype=float).reshape(-1, 3)
    v = np.asarray(v, dtype=float).reshape(-1, 3)
    w = np.asarray(omega, dtype=float).reshape(-1, 3)
    r = np.asarray(radius, dtype=float).reshape(-1)
    scale = resolution / box_size
    out = np.empty((len(r), 10))
    out[:, 0:3] = x * scale
    out[:, 3] = r * scale
    out[:, 4:7] = v * float(velocity_lu_scale)
    out[:, 7:10] = w * float(angular_lu_scale)
    return out


def lbm_converge(solver, residual_tol: float = 1.0e-8, min_steps: int = 1, max_steps: int = 20000,
                 check_every: int = 1):
    """Step until |mean_uz_k - mean_uz_{k-1}| / |mean_uz_k| < tol (couple_psc_liggghts.py:284-296).

    Returns (iterations, residual, converged, last diagnostics).  This package's solvers run the
    loop natively (``run_to_convergence``: the criterion on the device, loads and diagnostics of
    the stopping step only; ``check_every`` = k evaluates it every k steps, 1 = every step as the
    reference).  Any other object with the reference's ``collide_stream_psc()`` runs the
    reference's per-step loop (check_every must then be 1).
    """
    native = getattr(solver, "run_to_convergence", None)
    if native is not None:
        return native(residual_tol=residual_tol, min_steps=min_steps, max_steps=max_steps, check_every=check_every)
    if int(check_every) != 1:
        raise ValueError("check_every > 1 needs a solver of this package")
    previous = None
    residual = math.inf
    diag: dict = {}
    for iteration in range(1, int(max_steps) + 1):
        diag = solver.collide_stream_psc()
        current = float(diag.get("mean_uz", 0.0))
        if previous is not None:
            residual = abs(current - previous) / max(abs(current), 1.0e-30)
        previous = current
        if iteration >= min_steps and residual < residual_tol:
            return iteration, residual, True, diag
    return int(max_steps), residual, False, diag


def lbm_transient_advance(solver, steps: int):
    """Advance a fixed number of steps (couple_psc_liggghts.py:299-310)."""
    previous = float(np.mean(solver.uz))
    diag: dict = {}
    for _ in range(int(steps)):
        diag = solver.collide_stream_psc()
    current = float(diag.get("mean_uz", previous))
    residual = abs(current - previous) / max(abs(current), 1.0e-30)
    return int(steps), residual, True, diag


def loads_to_si(solver, force_scale: float, torque_scale: float, mask=None):
    """Forces / torques in SI, zeroed outside ``mask`` (couple_psc_liggghts.py:600-603)."""
    f = force_scale * np.asarray(solver.hydro_forces)
    t = torque_scale * np.asarray(solver.hydro_torques)
    if mask is not None:
        m = np.asarray(mask, dtype=bool)
        f[~m] = 0.0
        t[~m] = 0.0
    return f, t
