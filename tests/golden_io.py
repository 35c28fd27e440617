"""Loading helpers for the committed golden fixtures (produced by make_golden.py)."""

import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def names():
    """The PSC-IMB cases (psc3d.py)."""
    return sorted(p.stem for p in GOLDEN.glob("*.npz") if not p.stem.startswith("voxel_"))


def voxel_names():
    """The voxel bounce-back cases (run_3d_window_lbm.py)."""
    return sorted(p.stem for p in GOLDEN.glob("voxel_*.npz"))


def load(name):
    z = np.load(GOLDEN / f"{name}.npz")
    data = {k: z[k] for k in z.files}
    data["meta"] = json.loads(bytes(data["meta"]).decode())
    return data


def sparse_lists(data):
    counts = data["node_counts"]
    off = np.concatenate([[0], np.cumsum(counts)])
    ids = [data["node_ids"][off[i]:off[i + 1]] for i in range(len(counts))]
    vals = [data["alpha_vals"][off[i]:off[i + 1]] for i in range(len(counts))]
    return ids, vals


def rel_norm_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    num = np.linalg.norm(a - b)
    if den == 0.0:
        return num
    return num / den


def load_errors(forces, torques, ref_forces, ref_torques, radii):
    """(force error, torque error) as norm differences over a physical scale.

    Forces: relative to the reference force norm.  Torques: relative to the
    larger of the reference torque norm and |F| x (r + 1), because the torque
    of a symmetric body is pure round-off and has no meaningful own scale.
    """
    ref_forces = np.asarray(ref_forces, dtype=np.float64).reshape(-1, 3)
    ref_torques = np.asarray(ref_torques, dtype=np.float64).reshape(-1, 3)
    if ref_forces.size == 0:
        return 0.0, 0.0
    fnorm = float(np.linalg.norm(ref_forces))
    arm = float(np.linalg.norm(np.linalg.norm(ref_forces, axis=1) * (np.asarray(radii) + 1.0)))
    fe = float(np.linalg.norm(np.asarray(forces) - ref_forces)) / max(fnorm, 1e-300)
    te = float(np.linalg.norm(np.asarray(torques) - ref_torques)) / max(float(np.linalg.norm(ref_torques)), arm,
                                                                       1e-300)
    return fe, te
