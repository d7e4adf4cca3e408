"""The scenario builders against the reference's own (tests/golden/scenarios.json,
made by make_golden_scenarios.py): every field of the configuration they make
is equal, for the fixed-cylinder family at Re 20 / 40 / 100 / 200 with each
IB method, and for the oscillating cylinder."""
import json
import os

import pytest

from iblbm_b200.scenarios import make_dirichlet_neumann_fixed_cylinder_config, make_oscillating_cylinder_config

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "scenarios.json")) as f:
    G = json.load(f)


def _check(cfg, want):
    for k, v in want.items():
        assert hasattr(cfg, k), k
        got = getattr(cfg, k)
        assert (list(got) if isinstance(got, tuple) else got) == v, k


@pytest.mark.parametrize("k", range(len(G["fixed"])))
def test_fixed_cylinder_builder(k):
    args, want = G["fixed"][k]
    _check(make_dirichlet_neumann_fixed_cylinder_config(**args), want)


@pytest.mark.parametrize("k", range(len(G["oscillating"])))
def test_oscillating_cylinder_builder(k):
    args, want = G["oscillating"][k]
    _check(make_oscillating_cylinder_config(**args), want)


def test_fixed_cylinder_rejects_other_reynolds_numbers():
    with pytest.raises(ValueError):
        make_dirichlet_neumann_fixed_cylinder_config(reynolds=60)
