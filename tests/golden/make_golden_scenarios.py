"""Fixture for the scenario builders (tests/test_scenarios.py): the
configurations that the reference's own builders make
(scenarios/steady.py make_dirichlet_neumann_fixed_cylinder_config,
scenarios/oscillating.py make_oscillating_cylinder_config) for a set of
arguments, as JSON.

Usage:  python tests/golden/make_golden_scenarios.py --reference /path/to/reference
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

FIXED_ARGS = [dict(reynolds=re, ibm_method=m, delta_type=d, collision_model=c)
              for re in (20, 40, 100, 200) for m in ("DF", "MDF", "DFC")
              for d, c in (("hat", "BGK"), ("peskin4pt", "CM_MRT"))]
FIXED_ARGS += [dict(reynolds=40, ibm_method="MDF", max_steps=500, mdf_iterations=12, mdf_min_iterations=3, nn=201)]
OSC_ARGS = [dict(), dict(reynolds=40, kc=10.0, ibm_method="MDF", delta_type="hat", collision_model="TRT", nn=321,
                         max_steps=900)]


def _plain(cfg):
    return {k: v for k, v in dataclasses.asdict(cfg).items()
            if isinstance(v, (int, float, str, bool, type(None), tuple, list))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("IBLBM_REFERENCE"),
                    required="IBLBM_REFERENCE" not in os.environ,
                    help="reference checkout (or set IBLBM_REFERENCE)")
    args = ap.parse_args()
    os.environ["IBLBM_GPU"] = "0"
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/iblbm_numba_cache")
    sys.dont_write_bytecode = True
    sys.path.insert(0, args.reference)
    from scenarios.oscillating import make_oscillating_cylinder_config
    from scenarios.steady import make_dirichlet_neumann_fixed_cylinder_config
    out = {"fixed": [[a, _plain(make_dirichlet_neumann_fixed_cylinder_config(**a))] for a in FIXED_ARGS],
           "oscillating": [[a, _plain(make_oscillating_cylinder_config(**a))] for a in OSC_ARGS]}
    with open(os.path.join(HERE, "scenarios.json"), "w") as f:
        json.dump(out, f, sort_keys=True, separators=(",", ":"))
    print("wrote", os.path.join(HERE, "scenarios.json"))


if __name__ == "__main__":
    main()
