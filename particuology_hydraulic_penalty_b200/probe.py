"""Permeability probe on the GPU: LIGGGHTS dump in, one CSV row out.

Same command line, dump parsing, lattice scaling, Darcy quantities and CSV
schema as the reference's scripts/run_psc_permeability_resolution.py
(parse_dump :44-68, to_particles :71-76, filter :79-82, write_row :85-119,
main :122-192), so merge_permeability_convergence.py reads the rows
unchanged.  The solver is the drop-in SparsePscD3Q19 with an extra
``--precision`` (default fp64-exact, bit-identical to the reference) and
``--force-axis`` (default z, as in the reference).

    python -m particuology_hydraulic_penalty_b200.probe --case skeleton --resolution 64 \\
        --source-dump window.dump --steps 360 --outdir out/
"""

from __future__ import annotations

import argparse
import csv
from pathlib import Path

import numpy as np

BOX_SIZE_M = 9.0e-3

FIELDS = [
    "case", "resolution", "steps", "tau", "force_z", "subsamples", "geometry_workers", "source_dump",
    "particle_filter", "n_particles", "porosity_psc", "mean_uz_fluid", "superficial_uz", "max_uz",
    "permeability_lu", "K_over_skeleton_same_resolution", "momentum_residual", "particle_force_sum_x_lu",
    "particle_force_sum_y_lu", "particle_force_sum_z_lu", "particle_force_norm_sum_lu", "fluid_imb_sum_x_lu",
    "fluid_imb_sum_y_lu", "fluid_imb_sum_z_lu", "particle_fluid_momentum_closure_lu",
    "domain_body_force_z_lu", "fluid_volume_body_force_z_lu",
]


def parse_args(argv=None) -> argparse.Namespace:
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--case", required=True, choices=["skeleton", "baseline", "packed_slug"])
    p.add_argument("--resolution", type=int, required=True)
    p.add_argument("--source-dump", required=True)
    p.add_argument("--particle-filter", default="all", choices=["all", "type==1"])
    p.add_argument("--steps", type=int, default=360)
    p.add_argument("--tau", type=float, default=0.72)
    p.add_argument("--force-z", type=float, default=2.0e-7)
    p.add_argument("--subsamples", type=int, default=2)
    p.add_argument("--geometry-workers", type=int, default=1,
                   help="accepted for compatibility; voxelisation runs on the GPU")
    p.add_argument("--outdir", default="convergence/permeability")
    p.add_argument("--precision", default="fp64-exact", choices=["fp64-exact", "fp64", "fp32", "fp16", "bf16"])
    p.add_argument("--box-size-m", type=float, default=BOX_SIZE_M)
    p.add_argument("--quiet", action="store_true")
    return p.parse_args(argv)


def parse_dump(path: Path) -> np.ndarray:
    """Rows id, type, x, y, z, radius of a LIGGGHTS text dump (``ITEM: ATOMS`` section)."""
    lines = Path(path).read_text().splitlines()
    try:
        header = next(i for i, line in enumerate(lines) if line.startswith("ITEM: ATOMS"))
    except StopIteration:
        raise ValueError(f"{path} has no 'ITEM: ATOMS' section") from None
    cols = lines[header].split()[2:]
    idx = {name: i for i, name in enumerate(cols)}
    required = ["id", "type", "x", "y", "z", "radius"]
    missing = [name for name in required if name not in idx]
    if missing:
        raise ValueError(f"{path} missing dump columns: {missing}")
    rows = []
    for line in lines[header + 1:]:
        if not line.strip():
            continue
        if line.startswith("ITEM:"):
            break  # next timestep block
        parts = line.split()
        rows.append([int(float(parts[idx["id"]])), int(float(parts[idx["type"]])), float(parts[idx["x"]]),
                     float(parts[idx["y"]]), float(parts[idx["z"]]), float(parts[idx["radius"]])])
    return np.asarray(rows, dtype=float).reshape(-1, 6)


def filter_particles(rows: np.ndarray, particle_filter: str) -> np.ndarray:
    if particle_filter == "type==1":
        return rows[rows[:, 1] == 1]
    return rows


def to_particle_array(rows: np.ndarray, resolution: int, box_size_m: float = BOX_SIZE_M) -> np.ndarray:
    """(P, 10) particles in lattice units: positions and radii scaled by resolution / box size."""
    scale = resolution / box_size_m
    out = np.zeros((len(rows), 10))
    out[:, 0:3] = rows[:, 2:5] * scale
    out[:, 3] = rows[:, 5] * scale
    return out


def write_row(path: Path, row: dict) -> None:
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    with path.open("w", newline="") as f:
        writer = csv.DictWriter(f, fieldnames=FIELDS)
        writer.writeheader()
        writer.writerow(row)


def summarize(solver, args, n_rows: int, last: dict | None) -> dict:
    """The reference's CSV quantities from the final solver state (run_psc_permeability_resolution.py:144-190)."""
    fluid_weight = 1.0 - solver.solid
    fluid_volume = float(np.sum(fluid_weight))
    weighted_uz = solver.uz * fluid_weight
    mean_uz_fluid = float(np.sum(weighted_uz) / max(fluid_volume, 1.0e-300))
    superficial_uz = float(np.sum(weighted_uz) / solver.n ** 3)
    nu = (args.tau - 0.5) / 3.0
    permeability = float(nu * superficial_uz / max(args.force_z, 1.0e-300))
    pf = np.sum(solver.hydro_forces, axis=0) if len(solver.hydro_forces) else np.zeros(3)
    imb = np.array([float(np.sum(solver.imb_mx)), float(np.sum(solver.imb_my)), float(np.sum(solver.imb_mz))])
    return {
        "case": args.case, "resolution": args.resolution, "steps": args.steps, "tau": args.tau,
        "force_z": args.force_z, "subsamples": args.subsamples, "geometry_workers": args.geometry_workers,
        "source_dump": str(Path(args.source_dump).resolve()), "particle_filter": args.particle_filter,
        "n_particles": n_rows, "porosity_psc": fluid_volume / solver.n ** 3, "mean_uz_fluid": mean_uz_fluid,
        "superficial_uz": superficial_uz, "max_uz": float(np.max(solver.uz)), "permeability_lu": permeability,
        "K_over_skeleton_same_resolution": "",
        "momentum_residual": float(last["momentum_residual"] if last else np.nan),
        "particle_force_sum_x_lu": float(pf[0]), "particle_force_sum_y_lu": float(pf[1]),
        "particle_force_sum_z_lu": float(pf[2]), "particle_force_norm_sum_lu": float(np.linalg.norm(pf)),
        "fluid_imb_sum_x_lu": float(imb[0]), "fluid_imb_sum_y_lu": float(imb[1]), "fluid_imb_sum_z_lu": float(imb[2]),
        "particle_fluid_momentum_closure_lu": float(np.linalg.norm(pf + imb)),
        "domain_body_force_z_lu": float(args.force_z * solver.n ** 3),
        "fluid_volume_body_force_z_lu": float(args.force_z * fluid_volume),
    }


def main(argv=None) -> dict:
    from .psc3d import SparsePscD3Q19

    args = parse_args(argv)
    rows = filter_particles(parse_dump(Path(args.source_dump)), args.particle_filter)
    parts = to_particle_array(rows, args.resolution, args.box_size_m)
    solver = SparsePscD3Q19(n=args.resolution, particles=parts, tau=args.tau, subsamples=args.subsamples,
                            body_force_z=args.force_z, static_geometry=True, geometry_workers=args.geometry_workers,
                            precision=args.precision)
    last = None
    for step in range(args.steps):
        last = solver.collide_stream_psc()
        if not args.quiet and (step == 0 or (step + 1) % 60 == 0 or step + 1 == args.steps):
            print(f"{args.case} n={args.resolution} step={step + 1}/{args.steps} "
                  f"mean_uz={last['mean_uz']:.3e} residual={last['momentum_residual']:.3e}")
    row = summarize(solver, args, len(rows), last)
    out = Path(args.outdir) / f"{args.case}_n{args.resolution:03d}.csv"
    write_row(out, row)
    if not args.quiet:
        print(f"wrote {out}")
    return row


if __name__ == "__main__":
    main()
