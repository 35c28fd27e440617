"""Dump parsing and CSV schema of the GPU permeability probe (CPU parts)."""

import csv

import numpy as np
import pytest

from particuology_hydraulic_penalty_b200 import probe


DUMP = """ITEM: TIMESTEP
100
ITEM: NUMBER OF ATOMS
3
ITEM: BOX BOUNDS pp pp pp
0 0.009
0 0.009
0 0.009
ITEM: ATOMS id type x y z vx radius
1 1 0.0045 0.0045 0.0045 0 0.002
2 2 0.001 0.002 0.003 0 0.0003
3 1 0.008 0.0085 0.0001 0 0.0015
"""


def test_parse_dump_and_filter(tmp_path):
    p = tmp_path / "w.dump"
    p.write_text(DUMP)
    rows = probe.parse_dump(p)
    assert rows.shape == (3, 6)
    assert np.array_equal(rows[:, 0], [1, 2, 3]) and np.array_equal(rows[:, 1], [1, 2, 1])
    assert np.allclose(rows[:, 5], [0.002, 0.0003, 0.0015])
    assert probe.filter_particles(rows, "type==1").shape == (2, 6)


def test_missing_columns(tmp_path):
    p = tmp_path / "bad.dump"
    p.write_text("ITEM: ATOMS id type x y z\n1 1 0 0 0\n")
    with pytest.raises(ValueError, match="radius"):
        probe.parse_dump(p)


def test_scaling_to_lattice_units(tmp_path):
    p = tmp_path / "w.dump"
    p.write_text(DUMP)
    parts = probe.to_particle_array(probe.parse_dump(p), 64)
    # run_psc_permeability_resolution.py:71-76 scales by resolution / 9 mm
    assert np.allclose(parts[0, :4], [32.0, 32.0, 32.0, 0.002 * 64 / 9.0e-3])
    assert np.all(parts[:, 4:] == 0.0)


def test_csv_schema(tmp_path):
    row = {k: 0 for k in probe.FIELDS}
    out = tmp_path / "x" / "skeleton_n064.csv"
    probe.write_row(out, row)
    with out.open() as f:
        header = next(csv.reader(f))
    assert header == probe.FIELDS
    assert len(probe.FIELDS) == 27
