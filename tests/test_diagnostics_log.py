"""The diagnostics CSV against the reference's own writer, byte for byte.

sim::DiagnosticsLog (src/sim/diagnostics_log.cpp) writes a header row and one
row per measurement at 17 significant digits; the energy error is relative to
the first row (core::relative_energy_error, src/core/diagnostics.cpp:85-89),
the virial ratio is 2T/|U| (core/diagnostics.hpp:79-82). The same rows go
through the reference's class and through orrery_b200.DiagnosticsLog, and the
files must be identical; the rows include the degenerate cases both sides
define (no potential energy, nothing moving, a zero first energy) and numbers
at the ends of the double range. Runs on the CPU.
"""
from __future__ import annotations

import numpy as np
import pytest

from orrery_b200.simulation import DiagnosticsLog


def rows_from_states(reference, seed=5, count=4):
    rng = np.random.default_rng(seed)
    rows = []
    for r in range(count):
        n = 64
        x, y, z, vx, vy, vz = (rng.standard_normal(n) for _ in range(6))
        m = rng.uniform(0.5, 1.5, n) / n
        rows.append((r * 25, r * 25 * 1e-3, reference.diagnostics(x, y, z, vx, vy, vz, m, 0.01)))
    return rows


def row(step, time, kinetic, potential, linear=(0.0, 0.0, 0.0), angular=(0.0, 0.0, 0.0)):
    return (step, time, {"kinetic_energy": kinetic, "potential_energy": potential,
                         "linear_momentum": np.array(linear),
                         "angular_momentum": np.array(angular)})


def write_ours(path, rows):
    log = DiagnosticsLog(path)
    for step, time, d in rows:
        log.record(step, time, d)
    log.close()


CASES = {
    "measured": None,  # rows measured by core::measure_diagnostics
    "degenerate": [row(0, 0.0, 0.25, -0.5, (-0.0, 1e-300, -5e-324), (1e300, -2.5, 0.1)),
                   row(7, 7 * 0.003, 0.5, 0.0),            # virial ratio: infinity
                   row(8, 8 * 0.003, 0.0, 0.0),            # virial ratio: NaN (0/0)
                   row(1 << 40, 1.0e-7, 3.0, -1.0),
                   row(9, -0.0, 1.0 / 3.0, -2.0 / 3.0, (1.0 / 7.0, 2.0 / 7.0, 3.0 / 7.0))],
    "zero_first_energy": [row(0, 0.0, 0.5, -0.5), row(1, 0.001, 0.75, -0.5),
                          row(2, 0.002, 0.25, -0.75)],
    "empty": [],
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_rows_are_the_reference_writers_rows(reference, tmp_path, case):
    rows = CASES[case] if CASES[case] is not None else rows_from_states(reference)
    ours, theirs = tmp_path / "ours.csv", tmp_path / "theirs.csv"
    write_ours(ours, rows)
    reference.write_diagnostics_log(theirs, rows)
    assert ours.read_bytes() == theirs.read_bytes()
    assert ours.read_text().count("\n") == len(rows) + 1


def test_the_error_column_is_relative_to_the_first_row(tmp_path):
    path = tmp_path / "d.csv"
    write_ours(path, [row(0, 0.0, 0.25, -0.75), row(1, 0.1, 0.25, -0.7)])
    lines = path.read_text().splitlines()
    assert lines[0].split(",")[5] == "relative_energy_error"
    assert float(lines[1].split(",")[5]) == 0.0
    assert float(lines[2].split(",")[5]) == pytest.approx(0.05 / 0.5)
