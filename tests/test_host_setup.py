"""Host-side setup of the product (grid, tau, markers, MDF relaxation factor)
against the reference's golden values — CPU only."""
import os

import numpy as np
import pytest

from iblbm_b200.config import SimConfig
from iblbm_b200.physics import mdf_relaxation_factor, oscillation_table
from iblbm_b200.state import initialize

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def units():
    return dict(np.load(os.path.join(GOLD, "units.npz")))


@pytest.mark.parametrize("name", ["C1", "C2", "C3", "C5"])
def test_initialize_matches_reference(units, name):
    from tests.golden.make_golden import INIT_CASES
    st = initialize(SimConfig(**INIT_CASES[name]))
    got = np.array([st.nx, st.ny, st.dx, st.dy, st.tau, st.Larea, st.lattice_r, st.r, st.Lb], dtype=np.float64)
    np.testing.assert_array_equal(got, units[f"init_{name}_scal"])
    np.testing.assert_array_equal(st.Lx, units[f"init_{name}_Lx"])
    np.testing.assert_array_equal(st.Ly, units[f"init_{name}_Ly"])
    for p, part in enumerate(st.particles or []):
        np.testing.assert_array_equal(part.Lx, units[f"init_{name}_p{p}_Lx"])
        np.testing.assert_array_equal(np.array([part.mass, part.I_particle, part.Larea, part.Lb]),
                                      units[f"init_{name}_p{p}_scal"])


@pytest.mark.parametrize("delta", ["hat", "peskin4pt"])
def test_mdf_relaxation_factor_matches_reference(units, delta):
    om = mdf_relaxation_factor(units["i_Lx"], units["i_Ly"], delta, float(units["i_Larea"][0]),
                               float(units["i_dx"][0]))
    assert om == float(units[f"omega_{delta}"][0])


def test_mdf_relaxation_factor_config2():
    """Config 2 geometry (D = 40, P4): the reference's own value is 2.3737 to 4 digits."""
    from tests.golden.make_golden import INIT_CASES
    st = initialize(SimConfig(**INIT_CASES["C2"]))
    om = mdf_relaxation_factor(st.Lx, st.Ly, "peskin4pt", st.Larea, st.dx)
    assert abs(om - 2.3737) < 5e-4


def test_oscillation_table_matches_reference_motion():
    """Entry t + 1 is the displacement the reference sets after step t (motion.py)."""
    st = initialize(SimConfig(Re=100, NN=161, xmax=1, ymax=1, cylinder_center=(0.5, 0.5),
                              cylinder_D_ratio=0.125, lattice_u=0.02, inflow_u=0.0, motion_type="oscillating",
                              nx_formula="simple", bc_type="open_boundary"))
    tab = oscillation_table(50, 0.02, 5.0, st.r, st.lattice_r)
    f0 = 0.02 / (5.0 * 2.0 * st.lattice_r)
    A = 5.0 * 2.0 * st.r / (2.0 * np.pi)
    assert tab[1] == 0.0
    for t in (1, 7, 50):
        assert tab[t + 1] == A * np.sin(f0 * 2.0 * np.pi * t)


def test_pairwise_tree_reproduces_numpy_sum():
    """The summation tree the device uses for the particle forces: evaluated
    over only the nonzero entries of a sparse field, it equals np.sum of the
    dense field bit for bit (lattice sizes of the sedimentation runs and random
    ones; band-shaped and scattered nonzeros)."""
    import numpy as np
    from iblbm_b200.physics import pairwise_sum_sparse, pairwise_tree, pairwise_tree_index
    rng = np.random.default_rng(7)
    for n in (3, 64, 128, 129, 1000, 4097, 321 * 1281, 161 * 161):
        for _ in range(3):
            nb = int(rng.integers(1, min(n, 1500) + 1))
            idx = np.sort(rng.choice(n, nb, replace=False))
            val = rng.normal(size=nb) * 10.0 ** rng.integers(-6, 2)
            dense = np.zeros((n, 2))
            dense[idx, 0] = val
            assert pairwise_sum_sparse(n, idx, val) == dense[:, 0].sum()
        leaves, nodes, levels = pairwise_tree(n)
        lut, span = pairwise_tree_index(n, leaves, nodes)
        e = np.arange(n)
        leaf = np.searchsorted(leaves[:, 0], e, side="right") - 1
        assert np.all((leaf == lut[e // 64]) | (leaf == lut[e // 64] + 1))
        if len(nodes):
            assert tuple(span[-1]) == (0, len(leaves) - 1)
            assert levels[0] == 0 and levels[-1] == len(nodes)
