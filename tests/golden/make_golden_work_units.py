"""Writes work_units.json: the reference service's cost model evaluated by the
reference's own code (service/orrery_service/limits.py, work_units and
MAX_WORK), for cases the server's admission tests use.

    ORRERY_REFERENCE_ROOT=<reference checkout> python tests/golden/make_golden_work_units.py
"""
from __future__ import annotations

import importlib.util
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))


def main() -> None:
    root = os.environ.get("ORRERY_REFERENCE_ROOT")
    if not root:
        raise SystemExit("set ORRERY_REFERENCE_ROOT to the reference's checkout")
    limits_path = os.path.join(root, "service", "orrery_service", "limits.py")
    spec = importlib.util.spec_from_file_location("reference_limits", limits_path)
    limits = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(limits)
    cases = [(0, 10, "direct"), (1, 10, "barnes-hut"), (2, 7, "direct"), (1000, 20, "direct"),
             (1000, 20, "barnes-hut"), (20_000, 6_000, "barnes-hut"), (20_000, 6_000, "direct"),
             (4_000_000, 500, "barnes-hut"), (65_000, 2_000, "direct")]
    out = {"cases": [{"count": c, "steps": s, "solver": v, "work": limits.work_units(c, s, v)}
                     for c, s, v in cases],
           "MAX_WORK": limits.MAX_WORK, "MAX_PARTICLES": limits.MAX_PARTICLES}
    with open(os.path.join(HERE, "work_units.json"), "w") as fh:
        json.dump(out, fh, indent=1)


if __name__ == "__main__":
    main()
