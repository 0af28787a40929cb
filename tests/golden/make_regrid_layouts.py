"""Writes regrid_layouts.json: block layouts the compiled reference's
AMRHierarchy (amr.cpp:34-301, through oracle/ref_shim.cpp) produces for the
tracking-sphere scenarios of tests/test_regrid_cpu.py -- after initialize()
and after every sphere update and regrid of each scenario -- plus gradient
tagger counts (amr.cpp:653-731) on seeded Brill-Lindquist blocks.

    make -C oracle ref && python tests/golden/make_regrid_layouts.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from oracle.hierarchy import RefHierarchy  # noqa: E402

sys.path.insert(0, os.path.dirname(HERE))
from test_regrid_cpu import SCENARIOS, TAG_CASES, tag_case_state  # noqa: E402


def layout(rh):
    return [[lv, list(g.n), list(g.lo), list(g.hi)] for g, lv in zip(rh.geoms, rh.levels)]


def main():
    ref = oracle.Reference("strict")
    out = {"scenarios": [], "tags": []}
    for sc in SCENARIOS:
        rh = RefHierarchy(ref, sc["n"], sc["lo"], sc["hi"], sc["spheres"], sc["max_levels"])
        steps = [layout(rh)]
        for op, arg in sc["ops"]:
            if op == "update":
                rh.update_spheres(arg)
            else:
                rh.regrid(arg)
            steps.append(layout(rh))
        out["scenarios"].append(steps)
    for case in TAG_CASES:
        g, u = tag_case_state(case)
        out["tags"].append(ref.tag_count(g, u, case["var"], case["threshold"]))
    with open(os.path.join(HERE, "regrid_layouts.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
