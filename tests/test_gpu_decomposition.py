"""Slab decomposition on the CUDA path, ranks evaluated one after another in
one process (their all-reduce is a plain sum here): the owned-centre
energies and the forces summed over the slabs equal the whole-box call."""

import numpy as np
import pytest
import torch

from fennol_b200.decomposition import SlabPlan, rank_contribution
from fennol_b200.potential import HARTREE_TO_KCALMOL, ANIPotential
from fennol_b200.systems import water_box

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,ranks", [("fp32", 2), ("fp32", 3), ("bf16x2", 3)])
def test_slabs_sum_to_the_whole_box(cuda_device, precision, ranks):
    pot = ANIPotential(precision=precision, device=cuda_device, seed=0, bf16_weights=precision != "fp32")
    s = water_box(8, seed=43)  # 1536 atoms, 24.8 A cube
    e_ref, f_ref = pot.energy_and_forces(s.coordinates, s.species, [s.natoms], s.cell[None])
    f_ref = f_ref.double().cpu().numpy()
    plan = SlabPlan(s.cell, ranks, pot.aev_cfg.radial_cutoff)
    e_sum, f_sum = 0.0, np.zeros_like(f_ref)
    for r in range(ranks):
        e, f = rank_contribution(pot, plan, r, s.coordinates, s.species)
        e_sum += float(e)
        f_sum += f.cpu().numpy()
    de = abs(e_sum - float(e_ref.sum())) * HARTREE_TO_KCALMOL / s.natoms
    assert de < 1e-5, de
    scale = np.abs(f_ref).max()
    np.testing.assert_allclose(f_sum, f_ref, atol=2e-5 * scale, rtol=0)


def test_ghost_centres_carry_no_energy(cuda_device):
    """centres = 0 leaves only ghosts: zero energy and zero forces."""
    pot = ANIPotential(precision="fp32", device=cuda_device, seed=0)
    s = water_box(5, seed=44)
    e, f = pot.energy_and_forces(s.coordinates, s.species, [s.natoms], s.cell[None], centres=0)
    assert float(e.abs().sum()) == 0.0
    assert float(f.abs().max()) == 0.0
