"""Virial tensor through the adjoint (FeNNol's virial_tensor = dE/dS of the
deformation x -> x S, cell -> cell S) against strain autograd of the FP64
oracle, for periodic boxes (minimum image and periodic images) and molecules."""

import numpy as np
import pytest

from fennol_b200.fennix import FENNIX
from fennol_b200.params import AEVConfig, MLPConfig, init_weights, variables_to_weights
from fennol_b200.potential import ANIPotential
from fennol_b200.systems import molecule_batch, water_box
from oracle import ani_ref
from test_fennix_api import ani_modules, ani_preprocessing

pytestmark = pytest.mark.gpu
CFG, MCFG = AEVConfig(), MLPConfig()
REL = 2e-4  # of the largest virial component (float32 path vs FP64)


@pytest.fixture(scope="module")
def pot(cuda_device):
    return ANIPotential(precision="fp32", device=cuda_device, seed=0)


@pytest.mark.parametrize("n_side,seed", [(5, 1), (3, 2)])
def test_periodic_box_virial(pot, n_side, seed):
    s = water_box(n_side, seed=seed)   # 15.5 A: minimum image; 9.3 A: periodic images
    e, f, v = pot.energy_forces_virial(s.coordinates, s.species, [s.natoms], s.cell[None])
    r = ani_ref.energy_forces_virial(s.coordinates, s.species, [s.natoms], pot.weights, CFG, MCFG,
                                     cells=s.cell[None], minimum_image=n_side >= 5)
    v = v.cpu().numpy()
    np.testing.assert_allclose(v, r["virial"], rtol=0, atol=REL * np.abs(r["virial"]).max())


def test_molecule_virial_matches_positions_times_forces(pot):
    mols = molecule_batch(5, seed=23)
    xyz = np.concatenate([m.coordinates for m in mols])
    sp = np.concatenate([m.species for m in mols])
    nat = np.array([m.natoms for m in mols])
    e, f, v = pot.energy_forces_virial(xyz, sp, nat)
    r = ani_ref.energy_forces_virial(xyz, sp, nat, pot.weights, CFG, MCFG)
    v, f = v.cpu().numpy(), f.cpu().numpy().astype(np.float64)
    off = np.concatenate([[0], np.cumsum(nat)])
    for b in range(len(nat)):
        scale = np.abs(r["virial"][b]).max()
        np.testing.assert_allclose(v[b], r["virial"][b], rtol=0, atol=REL * scale)
        xf = -np.einsum("ia,ib->ab", xyz[off[b]:off[b + 1]], f[off[b]:off[b + 1]])
        np.testing.assert_allclose(v[b], xf, rtol=0, atol=REL * scale)


def test_virial_forces_equal_plain_call(pot):
    s = water_box(4, seed=3)
    e1, f1 = pot.energy_and_forces(s.coordinates, s.species, [s.natoms], s.cell[None])
    e1, f1 = e1.clone(), f1.clone()
    e2, f2, _ = pot.energy_forces_virial(s.coordinates, s.species, [s.natoms], s.cell[None])
    assert abs(float(e1[0]) - float(e2[0])) < 1e-9
    np.testing.assert_allclose(f1.cpu().numpy(), f2.cpu().numpy(), rtol=0, atol=1e-6)


def test_fennix_energy_and_forces_and_virial(cuda_device):
    s = water_box(5, seed=4)
    m = FENNIX(5.2, ani_modules(), ani_preprocessing(), energy_terms=["energy"], precision="fp32",
               rng_key=0)
    e, f, v, out = m.energy_and_forces_and_virial(species=s.species, coordinates=s.coordinates,
                                                 natoms=np.array([s.natoms]), cells=s.cell[None],
                                                 flags={"minimum_image": True})
    W = variables_to_weights([m.variables], CFG.species_order, "energy")
    r = ani_ref.energy_forces_virial(s.coordinates, s.species, [s.natoms], W, CFG, MCFG, cells=s.cell[None])
    assert out["virial_tensor"].shape == (1, 3, 3)
    np.testing.assert_allclose(v.cpu().numpy(), r["virial"], rtol=0, atol=REL * np.abs(r["virial"]).max())
