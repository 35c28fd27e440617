"""Generate the golden fixtures by running the reference kernel itself.

Usage (in a checkout that has the reference tree, NOT on a GPU host)::

    python tests/golden/make_golden.py --reference /path/to/particuology_Hydraulic-penalty-

It imports ``src/lbm_dem/psc3d.py`` from the reference tree (pure NumPy), runs
the cases listed in ``CASES`` and writes one compressed ``.npz`` per case
next to this script.  The fixtures pin both the CPU oracle
(``oracle/psc_oracle.py``) and the CUDA path; the tests never import the
reference.
"""

from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _particles(ref, rows):
    return [ref.Particle3D(*map(float, row)) for row in rows]


def _seeded_rows(seed, count, n, rmin, rmax, moving):
    rng = np.random.default_rng(seed)
    rows = []
    for _ in range(count):
        x, y, z = rng.uniform(-0.1 * n, 1.1 * n, size=3)
        r = rng.uniform(rmin, rmax)
        if moving:
            v = rng.normal(0.0, 1e-4, size=3)
            w = rng.normal(0.0, 2e-5, size=3)
        else:
            v = np.zeros(3)
            w = np.zeros(3)
        rows.append([x, y, z, r, *v, *w])
    return rows


# name -> dict(kind, n, rows, tau, subsamples, force_z, static, steps)
def cases():
    c = {}
    # The reference smoke test, tests/test_psc3d_smoke.py:6-23, run for 1 and 4 steps.
    c["smoke_n12"] = dict(kind="dense", n=12, rows=[[6.0, 6.0, 6.0, 2.0] + [0.0] * 6],
                          tau=0.72, subsamples=2, force_z=1.0e-7, static=True, steps=4)
    # Moving-sphere force check (20^3, r=2.5, u=(1e-4,0,0), tau=1, S=2, 100 steps),
    # the form run_d3q19_psc_moving_sphere_benchmark.py:62-129 uses.
    c["moving_sphere_n20"] = dict(kind="dense", n=20, rows=[[10.0, 10.0, 10.0, 2.5, 1.0e-4] + [0.0] * 5],
                                  tau=1.0, subsamples=2, force_z=0.0, static=False, steps=100)
    # Sparse packed window with overlapping, truncated, moving and spinning spheres;
    # S=3 (non-dyadic alphas, so the per-cell sum order matters).
    c["sparse_mixed_n16"] = dict(kind="sparse", n=16, rows=_seeded_rows(7, 9, 16, 1.2, 4.5, True),
                                 tau=0.8, subsamples=3, force_z=2.0e-7, static=False, steps=3)
    # Static sparse bed, S=4, body force, the permeability-probe form
    # (run_psc_permeability_resolution.py:127-143).
    c["sparse_static_n24"] = dict(kind="sparse", n=24, rows=_seeded_rows(11, 14, 24, 1.5, 5.5, False),
                                  tau=0.72, subsamples=4, force_z=2.0e-7, static=True, steps=6)
    # Dense, two overlapping spinning spheres, geometry rebuilt every step.
    c["dense_spin_n14"] = dict(kind="dense", n=14,
                               rows=[[6.3, 7.1, 6.8, 3.1, 2e-4, -1e-4, 5e-5, 1e-5, -3e-5, 2e-5],
                                     [8.9, 6.2, 7.4, 2.4, -1e-4, 3e-5, 0.0, 0.0, 4e-5, -1e-5]],
                               tau=0.9, subsamples=4, force_z=5.0e-7, static=False, steps=4)
    # Edge cases: one sphere fully outside the box (empty bbox), one straddling a face.
    c["edge_outside_n10"] = dict(kind="sparse", n=10,
                                 rows=[[-9.0, 4.0, 4.0, 2.0] + [0.0] * 6,
                                       [9.6, 5.0, 0.3, 2.2] + [0.0] * 6],
                                 tau=0.72, subsamples=2, force_z=1.0e-7, static=True, steps=2)
    # No particles at all.
    c["empty_n8"] = dict(kind="sparse", n=8, rows=[], tau=0.72, subsamples=2, force_z=1.0e-6,
                         static=True, steps=2)
    return c


def run_case(ref, spec):
    parts = _particles(ref, spec["rows"])
    if spec["kind"] == "dense":
        solver = ref.PscD3Q19(n=spec["n"], particles=parts, tau=spec["tau"], subsamples=spec["subsamples"],
                              body_force_z=spec["force_z"], static_geometry=spec["static"])
    else:
        solver = ref.SparsePscD3Q19(n=spec["n"], particles=parts, tau=spec["tau"],
                                    subsamples=spec["subsamples"], body_force_z=spec["force_z"],
                                    static_geometry=spec["static"])
    diags = []
    first = None
    for step in range(spec["steps"]):
        d = solver.collide_stream_psc()
        diags.append([d["solid_volume_lu"], d["mean_uz"], d["momentum_residual"], d["max_force"],
                      d["max_torque"]])
        if step == 0:
            first = dict(f=solver.f.copy(), hydro_forces=solver.hydro_forces.copy(),
                         hydro_torques=solver.hydro_torques.copy())
    out = dict(
        particles=np.asarray(spec["rows"], dtype=float).reshape(-1, 10),
        f=solver.f, solid=solver.solid, rho=solver.rho, ux=solver.ux, uy=solver.uy, uz=solver.uz,
        imb=np.stack([solver.imb_mx, solver.imb_my, solver.imb_mz]),
        hydro_forces=solver.hydro_forces, hydro_torques=solver.hydro_torques,
        momentum_residual=np.float64(solver.momentum_residual),
        diags=np.asarray(diags, dtype=float),
        hydro_forces_step1=first["hydro_forces"], hydro_torques_step1=first["hydro_torques"],
    )
    if spec["n"] <= 14:  # keep the committed fixtures small
        out["f_step1"] = first["f"]
    if spec["kind"] == "sparse":
        counts = np.array([len(i) for i in solver.node_ids], dtype=np.int64)
        out["node_ids"] = np.concatenate(solver.node_ids) if len(solver.node_ids) else np.zeros(0, np.int64)
        out["alpha_vals"] = np.concatenate(solver.alpha_vals) if len(solver.alpha_vals) else np.zeros(0)
        out["node_counts"] = counts
        out["alpha_sum_flat"] = solver.alpha_sum_flat
    else:
        out["alpha_p"] = solver.alpha_p
        out["owner_weights"] = solver.owner_weights
    meta = {k: spec[k] for k in ("kind", "n", "tau", "subsamples", "force_z", "static", "steps")}
    out["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    return out


def voxel_cases():
    """Cases of the reference's voxel bounce-back solver (scripts/run_3d_window_lbm.py)."""
    rng = np.random.default_rng(3)
    pts = rng.uniform(0.0, 0.009, size=(12, 3))
    return {
        "voxel_bb_n16": dict(points=pts, center=np.array([0.0045, 0.0045, 0.0045]),
                             size=np.array([0.009, 0.009, 0.009]), radius=0.0012, n=16, tau=0.8,
                             force_z=1e-6, steps=40),
        "voxel_bb_n12_offset": dict(points=pts[:5] + 0.001, center=np.array([0.005, 0.004, 0.0045]),
                                    size=np.array([0.008, 0.009, 0.007]), radius=0.0016, n=12, tau=0.72,
                                    force_z=2e-7, steps=25),
    }


def run_voxel_case(reference_root, spec):
    import types

    # The script imports matplotlib at module level for its figures; voxelize and
    # run_lbm do not use it, and it is not installed here: register a stub.
    if "matplotlib" not in sys.modules:
        mpl = types.ModuleType("matplotlib")
        mpl.pyplot = types.ModuleType("matplotlib.pyplot")
        sys.modules["matplotlib"] = mpl
        sys.modules["matplotlib.pyplot"] = mpl.pyplot
    sys.path.insert(0, str(Path(reference_root).resolve() / "scripts"))
    import run_3d_window_lbm as vref  # noqa: E402

    solid, dx = vref.voxelize(spec["points"], spec["center"], spec["size"], spec["radius"], spec["n"])
    res = vref.run_lbm(solid, spec["tau"], spec["force_z"], spec["steps"], return_fields=True)
    out = dict(points=spec["points"], center=spec["center"], size=spec["size"], solid=solid, dx=dx,
               ux=res["ux"], uy=res["uy"], uz=res["uz"],
               scalars=np.array([res["mean_uz_fluid"], res["superficial_uz"], res["max_uz"],
                                 res["permeability_lu"], res["porosity_voxel"]]))
    meta = {k: spec[k] for k in ("radius", "n", "tau", "force_z", "steps")}
    meta["kind"] = "voxel"
    out["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--reference", required=True, help="root of the reference checkout")
    ap.add_argument("--only", nargs="*", default=None)
    args = ap.parse_args()
    sys.path.insert(0, str(Path(args.reference).resolve()))
    from src.lbm_dem import psc3d as ref  # noqa: E402  (reference kernel, NumPy only)

    for name, spec in cases().items():
        if args.only and name not in args.only:
            continue
        out = run_case(ref, spec)
        np.savez_compressed(HERE / f"{name}.npz", **out)
        print(f"wrote {name}.npz")
    for name, spec in voxel_cases().items():
        if args.only and name not in args.only:
            continue
        out = run_voxel_case(args.reference, spec)
        np.savez_compressed(HERE / f"{name}.npz", **out)
        print(f"wrote {name}.npz")


if __name__ == "__main__":
    main()
