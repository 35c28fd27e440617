"""Precision and physics validation runs on the GPU.

The reference's validation campaign (validation/run_precision_validation.py),
with the same profiles, cases, stopping rule and summary rows, run through the
drop-in solver:

* ``run_settling``          single-particle settling against the Hasimoto-
                            corrected Stokes terminal speed (:236-322)
* ``run_hasimoto_case``     drag on a sphere moving through its periodic array,
                            normalised by Stokes drag and the Hasimoto
                            correction (:325-401)
* ``run_permeability_case`` Darcy permeability of a fixed periodic array against
                            the Hasimoto drag reference, plus the prescribed-
                            force balance (:404-507)
* ``PROFILES``              quick / standard / high grids (:82-126)
* ``should_stop``           steady-state stopping on the last 8 samples (:223-233)

Beyond the reference's campaign:

* ``precision_ladder`` -- the same windows run to steady state in FP64 and in
  the reduced storage modes; relative permeability error of each mode against
  FP64 (the deviation-storage claim: <= 1e-4).
* ``adjoint_check`` -- the adjoint permeability gradient against central
  differences and the FP64 adjoint, with its cost against the forward pass.

    python -m particuology_hydraulic_penalty_b200.validation profile --profile standard --out-dir DIR
    python -m particuology_hydraulic_penalty_b200.validation ladder --n 96 --tol 1e-8
"""

from __future__ import annotations

import argparse
import csv
import json
import time
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import windows as wgen
from .batch import PscBatch, WindowSpec


def hasimoto_factor(radius: float, box_length: float) -> float:
    """Periodic Stokes drag correction for a sphere in a cubic array (moving-sphere benchmark :50-54)."""
    lam = radius / box_length
    return float(1.0 / (1.0 - 2.837297 * lam + 4.19 * lam ** 3 - 27.4 * lam ** 6))


CS2 = 1.0 / 3.0
C_Z = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1], dtype=float)  # c_z, reference order


@dataclass(frozen=True)
class GridRun:
    n: int
    radius: float
    min_steps: int
    max_steps: int
    sample_every: int


@dataclass(frozen=True)
class Profile:
    subsamples: int
    target_re: float
    steady_tolerance: float
    force_balance_tolerance: float
    settling: GridRun
    hasimoto: tuple
    permeability: tuple


# The reference's validation profiles (validation/run_precision_validation.py:82-126), same values.
PROFILES = {
    "quick": Profile(2, 5.0e-3, 2.0e-2, 5.0e-2, GridRun(20, 2.5, 300, 800, 20),
                     (GridRun(20, 2.5, 300, 900, 30), GridRun(28, 3.5, 500, 1200, 40)),
                     (GridRun(20, 2.5, 600, 1800, 50),)),
    "standard": Profile(3, 5.0e-3, 1.0e-2, 2.0e-2, GridRun(32, 4.0, 800, 3000, 25),
                        (GridRun(24, 3.0, 900, 2400, 40), GridRun(32, 4.0, 1400, 4200, 50),
                         GridRun(40, 5.0, 2200, 6500, 60)),
                        (GridRun(24, 3.0, 1800, 5000, 60), GridRun(32, 4.0, 3000, 8500, 80),
                         GridRun(40, 5.0, 4500, 13000, 100))),
    "high": Profile(4, 2.5e-3, 5.0e-3, 1.0e-2, GridRun(48, 6.0, 3000, 10000, 50),
                    (GridRun(32, 4.0, 2500, 7000, 60), GridRun(48, 6.0, 5000, 15000, 100),
                     GridRun(64, 8.0, 9000, 26000, 140)),
                    (GridRun(32, 4.0, 5000, 14000, 100), GridRun(48, 6.0, 10000, 30000, 160),
                     GridRun(64, 8.0, 18000, 52000, 220))),
}

SUMMARY_FIELDS = ["case", "profile", "n", "radius_lu", "diameter_lu", "subsamples", "steps", "time_converged",
                  "reference_name", "reference_value", "measured_value", "signed_relative_error",
                  "absolute_relative_error", "steady_std_relative", "steady_drift_relative", "force_ratio_tail",
                  "effective_force_ratio_tail", "force_balance_relative", "force_balance_pass", "re_tail",
                  "hasimoto_lambda", "hasimoto_factor", "exact_porosity", "psc_porosity",
                  "solid_volume_relative_error", "momentum_residual_tail"]


def steady_metrics(values) -> tuple[float, float]:
    """Relative sample standard deviation and the relative drift between the two halves of a
    series (run_precision_validation.py:148-158)."""
    v = np.asarray(values, dtype=float)
    if len(v) < 2:
        return float("inf"), float("inf")
    scale = max(abs(float(np.mean(v))), 1.0e-30)
    std_rel = float(np.std(v, ddof=1) / scale)
    half = max(1, len(v) // 2)
    first, second = float(np.mean(v[:half])), float(np.mean(v[half:]))
    return std_rel, abs(second - first) / max(abs(second), 1.0e-30)


def should_stop(step: int, run: GridRun, values, steady_tolerance: float, extra_check=None) -> bool:
    """Steady when, past min_steps, the last 8 samples vary and drift by at most the tolerance
    (run_precision_validation.py:223-233)."""
    if step < run.min_steps or len(values) < 8:
        return False
    std_rel, drift_rel = steady_metrics(values[-8:])
    return std_rel <= steady_tolerance and drift_rel <= steady_tolerance and (extra_check is None or extra_check())


def geometry_metrics(n: int, radius: float, psc_porosity: float) -> tuple[float, float]:
    """Exact porosity of one sphere in n^3 and the relative error of the PSC solid volume."""
    exact_solid = 4.0 * np.pi * radius ** 3 / 3.0
    psc_solid = (1.0 - psc_porosity) * float(n ** 3)
    return 1.0 - exact_solid / float(n ** 3), abs(psc_solid - exact_solid) / exact_solid


def fluid_statistics(diag: dict, n: int) -> tuple[float, float, float]:
    """(intrinsic u_z, superficial u_z, porosity) of the fluid, weights 1 - solid
    (run_precision_validation.py:140-145), from the step's own FP64 reductions."""
    N = float(n ** 3)
    fluid = float(diag["fluid_volume_lu"])
    sup = float(diag["superficial_u"][2])
    return sup * N / max(fluid, 1.0e-30), sup, fluid / N


def summary_row(case, profile_name, run, subsamples, steps, time_converged, reference_name, reference_value,
                measured_value, std_rel, drift_rel, force_ratio_tail, effective_force_ratio_tail, force_balance_rel,
                force_balance_pass, re_tail, psc_porosity, momentum_residual_tail) -> dict:
    """One row of the campaign's summary table (the reference's common_summary fields, :169-220)."""
    exact_porosity, volume_error = geometry_metrics(run.n, run.radius, psc_porosity)
    signed = measured_value / max(reference_value, 1.0e-30) - 1.0
    return {"case": case, "profile": profile_name, "n": run.n, "radius_lu": run.radius,
            "diameter_lu": 2.0 * run.radius, "subsamples": subsamples, "steps": steps,
            "time_converged": int(time_converged), "reference_name": reference_name,
            "reference_value": reference_value, "measured_value": measured_value, "signed_relative_error": signed,
            "absolute_relative_error": abs(signed), "steady_std_relative": std_rel, "steady_drift_relative": drift_rel,
            "force_ratio_tail": force_ratio_tail, "effective_force_ratio_tail": effective_force_ratio_tail,
            "force_balance_relative": force_balance_rel, "force_balance_pass": force_balance_pass,
            "re_tail": re_tail, "hasimoto_lambda": run.radius / float(run.n),
            "hasimoto_factor": hasimoto_factor(run.radius, float(run.n)), "exact_porosity": exact_porosity,
            "psc_porosity": psc_porosity, "solid_volume_relative_error": volume_error,
            "momentum_residual_tail": momentum_residual_tail}


def run_settling(profile_name: str, profile: Profile, tau: float = 0.72, density_ratio: float = 2.5,
                 precision: str = "fp64-exact") -> dict:
    """A free sphere under an external force settles through its periodic array; its terminal speed
    relative to the fluid against the Hasimoto-corrected Stokes speed (:236-322).  The geometry is
    voxelised again every step as the sphere moves (on the GPU)."""
    from .psc3d import Particle3D, PscD3Q19

    run = profile.settling
    nu = CS2 * (tau - 0.5)
    ref_speed = profile.target_re * nu / (2.0 * run.radius)
    external = -6.0 * np.pi * nu * run.radius * hasimoto_factor(run.radius, float(run.n)) * ref_speed
    mass = density_ratio * 4.0 * np.pi * run.radius ** 3 / 3.0
    sphere = Particle3D(0.5 * run.n, 0.5 * run.n, 0.5 * run.n, run.radius)
    solver = PscD3Q19(run.n, [sphere], tau=tau, subsamples=profile.subsamples, precision=precision)
    speeds, nets, resid = [], [], []
    porosity, last = float("nan"), 0
    for step in range(1, run.max_steps + 1):
        diag = solver.collide_stream_psc()
        hydro = float(solver.hydro_forces[0, 2])
        net = external + hydro
        sphere.vz += net / mass
        sphere.z = (sphere.z + sphere.vz) % float(run.n)
        last = step
        if step % run.sample_every == 0 or step == run.max_steps:
            intrinsic, _, porosity = fluid_statistics(solver.step_diagnostics(), run.n)
            speeds.append(abs(sphere.vz - intrinsic))
            nets.append(net)
            resid.append(float(diag["momentum_residual"]))
            if should_stop(step, run, speeds, profile.steady_tolerance,
                           lambda: abs(float(np.mean(nets[-8:]))) / abs(external) <= profile.force_balance_tolerance):
                break
    tail = min(8, len(speeds))
    std_rel, drift_rel = steady_metrics(speeds[-tail:])
    balance = abs(float(np.mean(nets[-tail:]))) / abs(external)
    ratio = abs(float(np.mean(nets[-tail:])) - external) / abs(external)
    conv = std_rel <= profile.steady_tolerance and drift_rel <= profile.steady_tolerance
    mean_speed = float(np.mean(speeds[-tail:]))
    return summary_row("single_particle_settling", profile_name, run, profile.subsamples, last, conv,
                       "Hasimoto-corrected Stokes terminal relative speed", ref_speed, mean_speed, std_rel, drift_rel,
                       ratio, float("nan"), balance, int(balance <= profile.force_balance_tolerance),
                       2.0 * run.radius * mean_speed / nu, porosity, float(np.mean(resid[-tail:])))


def _advance_to(solver, step: int, sample_every: int, max_steps: int):
    """Steps up to the next sampling step (step % sample_every == 0, or max_steps) in one call."""
    nxt = min(((step // sample_every) + 1) * sample_every, max_steps)
    return nxt, nxt - step


def run_hasimoto_case(profile_name: str, profile: Profile, run: GridRun, tau: float = 0.72,
                      precision: str = "fp64-exact") -> dict:
    """Resistance of a sphere moving at a fixed velocity through its periodic array, Stokes drag times
    the Hasimoto factor as the reference (:325-401).  The steps between samples run as one native
    call (the populations are those of single steps; the loads are read only at samples)."""
    from .psc3d import Particle3D, PscD3Q19

    nu = CS2 * (tau - 0.5)
    corr = hasimoto_factor(run.radius, float(run.n))
    u = profile.target_re * nu / (2.0 * run.radius)
    sphere = Particle3D(0.5 * run.n, 0.5 * run.n, 0.5 * run.n, run.radius, vz=u)
    solver = PscD3Q19(run.n, [sphere], tau=tau, subsamples=profile.subsamples, static_geometry=True,
                      precision=precision)
    ratios, resid, res = [], [], []
    porosity, step = float("nan"), 0
    while step < run.max_steps:
        step, k = _advance_to(solver, step, run.sample_every, run.max_steps)
        diag = solver.advance(k)
        intrinsic, _, porosity = fluid_statistics(solver.step_diagnostics(), run.n)
        rel = u - intrinsic
        fz = float(solver.hydro_forces[0, 2])
        ratios.append(abs(fz) / max(6.0 * np.pi * nu * run.radius * abs(rel), 1.0e-30) / corr)
        resid.append(float(diag["momentum_residual"]))
        res.append(2.0 * run.radius * abs(rel) / nu)
        if should_stop(step, run, ratios, profile.steady_tolerance):
            break
    tail = min(8, len(ratios))
    std_rel, drift_rel = steady_metrics(ratios[-tail:])
    conv = std_rel <= profile.steady_tolerance and drift_rel <= profile.steady_tolerance
    return summary_row("periodic_moving_sphere_hasimoto", profile_name, run, profile.subsamples, step, conv,
                       "Hasimoto-normalized resistance ratio", 1.0, float(np.mean(ratios[-tail:])), std_rel,
                       drift_rel, float("nan"), float("nan"), float("nan"), "", float(np.mean(res[-tail:])), porosity,
                       float(np.mean(resid[-tail:])))


def run_permeability_case(profile_name: str, profile: Profile, run: GridRun, tau: float = 0.72,
                          precision: str = "fp64-exact") -> dict:
    """Darcy permeability of a fixed sphere's periodic array driven by a body force, against
    K_ref = phi n^3 / (6 pi r Hasimoto factor) (:404-507, the formula at :421), with the balance of
    the particle force against the imposed force.  The fluid momentum change of a sampled step comes
    from the populations before and after it."""
    from .psc3d import Particle3D, PscD3Q19

    nu = CS2 * (tau - 0.5)
    corr = hasimoto_factor(run.radius, float(run.n))
    target = profile.target_re * nu / (2.0 * run.radius)
    body = target * 6.0 * np.pi * nu * run.radius * corr / float(run.n ** 3)
    sphere = Particle3D(0.5 * run.n, 0.5 * run.n, 0.5 * run.n, run.radius)
    solver = PscD3Q19(run.n, [sphere], tau=tau, subsamples=profile.subsamples, body_force_z=body,
                      static_geometry=True, precision=precision)
    exact_porosity, _ = geometry_metrics(run.n, run.radius, 1.0)
    k_ref = exact_porosity * run.n ** 3 / (6.0 * np.pi * run.radius * corr)
    expected = body * run.n ** 3
    cz = C_Z[:, None, None, None]
    perms, balances, ratios, eff_ratios, res, resid = [], [], [], [], [], []
    porosity, step = float("nan"), 0
    while step < run.max_steps:
        step, k = _advance_to(solver, step, run.sample_every, run.max_steps)
        if k > 1:
            solver.advance(k - 1)
        before = float(np.sum(solver.f * cz))
        diag = solver.collide_stream_psc()
        after = float(np.sum(solver.f * cz))
        intrinsic, superficial, porosity = fluid_statistics(solver.step_diagnostics(), run.n)
        fz = float(solver.hydro_forces[0, 2])
        perms.append(nu * superficial / body)
        balances.append(abs(abs(fz) - expected) / expected)
        ratios.append(abs(fz) / expected)
        eff_ratios.append((after - before + fz) / expected)
        res.append(2.0 * run.radius * abs(intrinsic) / nu)
        resid.append(float(diag["momentum_residual"]))
        if should_stop(step, run, perms, profile.steady_tolerance):
            break
    tail = min(8, len(perms))
    std_rel, drift_rel = steady_metrics(perms[-tail:])
    balance = float(np.mean(balances[-tail:]))
    conv = std_rel <= profile.steady_tolerance and drift_rel <= profile.steady_tolerance
    return summary_row("periodic_fixed_array_permeability", profile_name, run, profile.subsamples, step, conv,
                       "Darcy permeability from Hasimoto periodic drag", k_ref, float(np.mean(perms[-tail:])),
                       std_rel, drift_rel, float(np.mean(ratios[-tail:])), float(np.mean(eff_ratios[-tail:])),
                       balance, int(balance <= profile.force_balance_tolerance), float(np.mean(res[-tail:])),
                       porosity, float(np.mean(resid[-tail:])))


def run_profile(profile_name: str = "quick", cases=("settling", "hasimoto", "permeability"), tau: float = 0.72,
                density_ratio: float = 2.5, precision: str = "fp64-exact", out_dir=None) -> list[dict]:
    """Every selected case of one profile; with out_dir, the summary table as CSV and a report."""
    prof = PROFILES[profile_name]
    rows = []
    t0 = time.time()
    if "settling" in cases:
        rows.append(run_settling(profile_name, prof, tau, density_ratio, precision))
    if "hasimoto" in cases:
        rows += [run_hasimoto_case(profile_name, prof, run, tau, precision) for run in prof.hasimoto]
    if "permeability" in cases:
        rows += [run_permeability_case(profile_name, prof, run, tau, precision) for run in prof.permeability]
    if out_dir is not None:
        out = Path(out_dir)
        out.mkdir(parents=True, exist_ok=True)
        with (out / "precision_error_table.csv").open("w", newline="") as fh:
            w = csv.DictWriter(fh, fieldnames=SUMMARY_FIELDS)
            w.writeheader()
            w.writerows(rows)
        lines = [f"# PSC-IMB precision validation (GPU, precision {precision})", "", f"Profile: `{profile_name}`, "
                 f"{time.time() - t0:.1f} s", "",
                 "| case | N | d/lattice | steps | time converged | measured/reference | abs. relative error | "
                 "steady drift | force balance |", "|---|---:|---:|---:|---:|---:|---:|---:|---:|"]
        for r in rows:
            ratio = float(r["measured_value"]) / max(float(r["reference_value"]), 1.0e-30)
            lines.append(f"| {r['case']} | {r['n']} | {r['diameter_lu']:.4f} | {r['steps']} | {r['time_converged']} | "
                         f"{ratio:.6f} | {r['absolute_relative_error']:.4e} | {r['steady_drift_relative']:.4e} | "
                         f"{float(r['force_balance_relative']):.4e} |")
        (out / "precision_validation_report.md").write_text("\n".join(lines) + "\n")
    return rows


def precision_ladder(windows, precisions=("fp64", "fp32", "fp16", "bf16"), tau: float = 0.8,
                     force=(1.0e-6, 0.0, 0.0), subsamples: int = 4, tol: float = 1.0e-8, check_every: int = 200,
                     max_steps: int = 100000) -> dict:
    specs = [WindowSpec(w.n, w.particles, tau, tuple(force), subsamples, getattr(w, "kind", "")) for w in windows]
    out = {}
    for prec in precisions:
        t0 = time.time()
        b = PscBatch(specs, precision=prec, graph_steps=20)
        res = b.run_to_convergence(tol=tol, check_every=check_every, max_steps=max_steps)
        out[prec] = {"permeability": res["permeability"].tolist(), "steps": res["steps"].tolist(),
                     "residual": res["residual"].tolist(), "converged": res["converged"].tolist(),
                     "wall_s": time.time() - t0}
        del b
    ref = np.asarray(out[precisions[0]]["permeability"])
    for prec in precisions[1:]:
        k = np.asarray(out[prec]["permeability"])
        out[prec]["rel_err_vs_" + precisions[0]] = (np.abs(k - ref) / np.abs(ref)).tolist()
    return out


def hasimoto_drag(n: int = 32, radius: float = 4.0, tau: float = 1.0, subsamples: int = 4, velocity: float = 1e-4,
                  steps: int = 4000, precision: str = "fp64") -> dict:
    """Steady drag ratio |F| / (6 pi nu r |u_rel|) / Hasimoto factor for a sphere moving along x."""
    from .psc3d import Particle3D, PscD3Q19

    sphere = [Particle3D(0.5 * n, 0.5 * n, 0.5 * n, radius, vx=velocity)]
    s = PscD3Q19(n=n, particles=sphere, tau=tau, subsamples=subsamples, static_geometry=True, precision=precision)
    nu = (tau - 0.5) / 3.0
    hist = []
    for k in range(steps):
        s.collide_stream_psc()
        if (k + 1) % max(1, steps // 20) == 0:
            fluid = 1.0 - s.solid
            mean_ux = float(np.sum(fluid * s.ux) / max(float(np.sum(fluid)), 1e-30))
            fx = float(s.hydro_forces[0, 0])
            rel = velocity - mean_ux
            ratio = abs(fx) / (6.0 * np.pi * nu * radius * max(abs(rel), 1e-30))
            hist.append(ratio)
    tail = np.asarray(hist[len(hist) // 2:])
    h = hasimoto_factor(radius, float(n))
    return {"n": n, "radius": radius, "tau": tau, "ratio_tail": float(tail.mean()),
            "ratio_over_hasimoto": float(tail.mean() / h), "hasimoto_factor": h}


def adjoint_check(n: int = 96, n_fines: int = 64, steps: int = 2000, every: int = 100, n_check: int = 8,
                  h: float = 1.0e-3, seed: int = 5, eps: float = 0.05, tau: float = 0.8,
                  force=(1.0e-6, 0.0, 0.0), subsamples: int = 4) -> dict:
    """Adjoint dK/d(x, y, z, r) of the fines of a preloaded window vs central differences.

    The FP32 adjoint (the production setting) is timed against its forward
    pass; its gradient is compared with the FP64 adjoint and with FP64
    central differences of K for ``n_check`` seeded random fines.  The
    gradient of a fine sums over its periodic images (all emitted copies).
    """
    import torch

    from .adjoint import PermeabilityProblem

    w = wgen.make_window(n, "preloaded", seed, n_fines=n_fines)
    parts = w.particles
    fines = np.unique(w.owner[w.is_fine])
    rng = np.random.default_rng(seed)
    pick = rng.choice(fines, size=min(n_check, len(fines)), replace=False)

    def problem(prec):
        return PermeabilityProblem(n, tau=tau, force=force, subsamples=subsamples, eps=eps, steps=steps,
                                   checkpoint_every=every, precision=prec)

    def per_sphere(g):
        out = np.zeros((w.n_spheres, 4))
        np.add.at(out, w.owner, g)
        return out

    p32 = problem("fp32")
    p32.forward(parts)  # untimed: first launches, buffers
    p32.backward()
    # two timed forward + backward passes, the faster of each kept (a pass is thousands of launches,
    # so host noise shows in a single measurement)
    t_fwd = t_bwd = float("inf")
    for _ in range(2):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize()
        ev[0].record()
        K32 = p32.forward(parts)
        ev[1].record()
        g32 = per_sphere(p32.backward())
        ev[2].record()
        torch.cuda.synchronize()
        t_fwd = min(t_fwd, ev[0].elapsed_time(ev[1]) * 1e-3)  # CUDA events on the current stream (the handle
        t_bwd = min(t_bwd, ev[1].elapsed_time(ev[2]) * 1e-3)  # synchronises)
    p64 = problem("fp64")
    K64 = p64.forward(parts)
    g64 = per_sphere(p64.backward())
    gap = p64.solid_gap()
    rows = []
    for s_id in pick:
        idx = np.nonzero(w.owner == s_id)[0]
        for k in range(4):
            pp = parts.copy()
            pp[idx, k] += h
            pm = parts.copy()
            pm[idx, k] -= h
            fd = (problem("fp64").forward(pp) - problem("fp64").forward(pm)) / (2.0 * h)
            rows.append({"sphere": int(s_id), "component": "xyzr"[k], "fd_fp64": fd, "adjoint_fp64": g64[s_id, k],
                         "adjoint_fp32": g32[s_id, k]})
    fd = np.array([r["fd_fp64"] for r in rows])
    a64 = np.array([r["adjoint_fp64"] for r in rows])
    a32 = np.array([r["adjoint_fp32"] for r in rows])
    scale = np.abs(fd).max()
    return {
        "n": n, "steps": steps, "checkpoint_every": every, "n_fines": int(len(fines)), "K_fp32": K32,
        "K_fp64": K64, "forward_s_fp32": t_fwd, "backward_s_fp32": t_bwd, "backward_over_forward": t_bwd / t_fwd,
        "adjoint_plus_forward_over_forward": (t_fwd + t_bwd) / t_fwd,
        "fd_vs_adjoint_fp64_max_rel": float(np.max(np.abs(fd - a64) / np.maximum(np.abs(fd), 1e-3 * scale))),
        "fd_vs_adjoint_fp64_norm_rel": float(np.linalg.norm(fd - a64) / np.linalg.norm(fd)),
        "adjoint_fp32_vs_fp64_norm_rel": float(np.linalg.norm(a32 - a64) / np.linalg.norm(a64)),
        "fd_vs_adjoint_fp32_norm_rel": float(np.linalg.norm(fd - a32) / np.linalg.norm(fd)),
        "solid_gap_smooth_vs_counted": gap, "checks": rows,
    }


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = ap.add_subparsers(dest="cmd", required=True)
    lad = sub.add_parser("ladder")
    lad.add_argument("--n", type=int, default=96)
    lad.add_argument("--seed", type=int, default=1000)
    lad.add_argument("--tol", type=float, default=1e-8)
    lad.add_argument("--check-every", type=int, default=200)
    lad.add_argument("--max-steps", type=int, default=100000)
    lad.add_argument("--precisions", nargs="+", default=["fp64", "fp32", "fp16", "bf16"])
    lad.add_argument("--kinds", nargs="+", default=list(wgen.GEOMETRY_TYPES))
    lad.add_argument("--sizes", nargs="+", type=int, default=None, help="window edges (default: --n)")
    adj = sub.add_parser("adjoint")
    adj.add_argument("--n", type=int, default=96)
    adj.add_argument("--fines", type=int, default=64)
    adj.add_argument("--steps", type=int, default=2000)
    adj.add_argument("--every", type=int, default=100)
    adj.add_argument("--check", type=int, default=8)
    prof = sub.add_parser("profile", help="the reference's validation campaign (settling, Hasimoto, permeability)")
    prof.add_argument("--profile", choices=tuple(PROFILES), default="quick")
    prof.add_argument("--case", choices=("all", "settling", "hasimoto", "permeability"), default="all")
    prof.add_argument("--tau", type=float, default=0.72)
    prof.add_argument("--particle-density-ratio", type=float, default=2.5)
    prof.add_argument("--precision", default="fp64-exact")
    prof.add_argument("--out-dir", default=None)
    has = sub.add_parser("hasimoto")
    has.add_argument("--n", type=int, default=32)
    has.add_argument("--radius", type=float, default=4.0)
    has.add_argument("--steps", type=int, default=4000)
    args = ap.parse_args(argv)
    if args.cmd == "ladder":
        wins = [wgen.make_window(n, k, args.seed) for n in (args.sizes or [args.n]) for k in args.kinds]
        res = precision_ladder(wins, precisions=tuple(args.precisions), tol=args.tol, check_every=args.check_every,
                               max_steps=args.max_steps)
    elif args.cmd == "profile":
        cases = ("settling", "hasimoto", "permeability") if args.case == "all" else (args.case,)
        res = run_profile(args.profile, cases, tau=args.tau, density_ratio=args.particle_density_ratio,
                          precision=args.precision, out_dir=args.out_dir)
    elif args.cmd == "adjoint":
        res = adjoint_check(n=args.n, n_fines=args.fines, steps=args.steps, every=args.every, n_check=args.check)
    else:
        res = hasimoto_drag(n=args.n, radius=args.radius, steps=args.steps)
    print(json.dumps(res))
    return res


if __name__ == "__main__":
    main()
