"""Precision and physics validation runs on the GPU.

* ``precision_ladder`` -- the same windows run to steady state in FP64 and
  in the reduced storage modes; relative permeability error of each mode
  against FP64 (the deviation-storage claim: <= 1e-4).
* ``hasimoto_drag`` -- drag on a sphere moving through a periodic array,
  normalised by Stokes drag and the Hasimoto periodic correction, the check
  of scripts/run_d3q19_psc_moving_sphere_benchmark.py:50-129 and
  validation/run_precision_validation.py:325-401.

    python -m particuology_hydraulic_penalty_b200.validation ladder --n 96 --tol 1e-8
"""

from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import windows as wgen
from .batch import PscBatch, WindowSpec


def hasimoto_factor(radius: float, box_length: float) -> float:
    """Periodic Stokes drag correction for a sphere in a cubic array (moving-sphere benchmark :50-54)."""
    lam = radius / box_length
    return float(1.0 / (1.0 - 2.837297 * lam + 4.19 * lam ** 3 - 27.4 * lam ** 6))


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
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    K32 = p32.forward(parts)
    torch.cuda.synchronize()
    t_fwd = time.perf_counter() - t0
    t0 = time.perf_counter()
    g32 = per_sphere(p32.backward())
    torch.cuda.synchronize()
    t_bwd = time.perf_counter() - t0
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
    has = sub.add_parser("hasimoto")
    has.add_argument("--n", type=int, default=32)
    has.add_argument("--radius", type=float, default=4.0)
    has.add_argument("--steps", type=int, default=4000)
    args = ap.parse_args(argv)
    if args.cmd == "ladder":
        wins = [wgen.make_window(n, k, args.seed) for n in (args.sizes or [args.n]) for k in args.kinds]
        res = precision_ladder(wins, precisions=tuple(args.precisions), tol=args.tol, check_every=args.check_every,
                               max_steps=args.max_steps)
    elif args.cmd == "adjoint":
        res = adjoint_check(n=args.n, n_fines=args.fines, steps=args.steps, every=args.every, n_check=args.check)
    else:
        res = hasimoto_drag(n=args.n, radius=args.radius, steps=args.steps)
    print(json.dumps(res))
    return res


if __name__ == "__main__":
    main()
