"""Golden summaries of the reference's precision-validation cases, made by running the reference.

Usage (in a checkout that has the reference tree, NOT on a GPU host)::

    python tests/golden/make_validation_golden.py --reference /path/to/particuology_Hydraulic-penalty-

It imports ``validation/run_precision_validation.py`` from the reference tree
(NumPy; the plotting module its helper script imports at module level is
replaced by an empty stub, none of the functions used here draws) and runs the
``quick`` profile of each case with the script's defaults (tau 0.72, particle
density ratio 2.5):

* ``run_settling``            single-particle settling (:236-322)
* ``run_hasimoto_case``       both Hasimoto grids (:325-401)
* ``run_permeability_case``   fixed-array permeability (:404-507)

and writes their summary rows to ``validation_quick.json`` next to this
script.  The GPU validation harness must reproduce these rows.
"""

from __future__ import annotations

import argparse
import json
import sys
import tempfile
import types
from pathlib import Path

HERE = Path(__file__).resolve().parent


def main():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--reference", required=True, help="root of the reference checkout")
    ap.add_argument("--profile", default="quick")
    args = ap.parse_args()
    if "matplotlib" not in sys.modules:
        mpl = types.ModuleType("matplotlib")
        mpl.use = lambda *a, **k: None
        mpl.pyplot = types.ModuleType("matplotlib.pyplot")
        sys.modules["matplotlib"] = mpl
        sys.modules["matplotlib.pyplot"] = mpl.pyplot
    root = Path(args.reference).resolve()
    sys.path.insert(0, str(root))
    sys.path.insert(0, str(root / "validation"))
    import run_precision_validation as rpv  # noqa: E402  (the reference's validation driver)

    prof = rpv.PROFILES[args.profile]
    tau, density_ratio = 0.72, 2.5
    rows = []
    with tempfile.TemporaryDirectory() as tmp:
        out = Path(tmp)
        rows.append(rpv.run_settling(out, args.profile, prof, tau, density_ratio))
        print("settling", rows[-1]["steps"], rows[-1]["measured_value"], flush=True)
        for run in prof.hasimoto:
            rows.append(rpv.run_hasimoto_case(out, args.profile, prof, tau, run))
            print("hasimoto", run.n, rows[-1]["steps"], rows[-1]["measured_value"], flush=True)
        for run in prof.permeability:
            rows.append(rpv.run_permeability_case(out, args.profile, prof, tau, run))
            print("permeability", run.n, rows[-1]["steps"], rows[-1]["measured_value"], flush=True)
    meta = {"profile": args.profile, "tau": tau, "particle_density_ratio": density_ratio,
            "source": "validation/run_precision_validation.py of the reference, run by this script"}
    (HERE / f"validation_{args.profile}.json").write_text(json.dumps({"meta": meta, "rows": rows}, indent=1) + "\n")
    print(f"wrote validation_{args.profile}.json")


if __name__ == "__main__":
    main()
