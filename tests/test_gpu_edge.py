"""Edge cases of the energy/force path: isolated atoms (empty neighbour rows),
one-atom and empty systems inside a batch, an empty batch, and a single
species absent from a batch."""

import numpy as np
import pytest
import torch

from fennol_b200.params import AEVConfig, MLPConfig
from fennol_b200.potential import ANIPotential, HARTREE_TO_KCALMOL
from fennol_b200.systems import molecule_batch
from oracle import ani_ref

pytestmark = pytest.mark.gpu
CFG, MCFG = AEVConfig(), MLPConfig()


@pytest.fixture(scope="module")
def pot(cuda_device):
    return ANIPotential(precision="fp32", device=cuda_device, seed=0)


@pytest.fixture(scope="module")
def pot_tc(cuda_device):
    return ANIPotential(precision="bf16x2", bf16_weights=True, device=cuda_device, seed=0)


def check(pot, xyz, sp, nat, tol_e=1e-4, tol_f=0.05):
    e, f = pot.energy_and_forces(xyz, sp, nat)
    r = ani_ref.energy_and_forces(xyz, sp, nat, pot.weights, CFG, MCFG)
    nat = np.asarray(nat)
    de = np.abs(e.cpu().numpy() - r["energy"]) * HARTREE_TO_KCALMOL / np.maximum(nat, 1)
    assert de.max() <= tol_e, de
    if xyz.shape[0]:
        rmse = np.sqrt(np.mean((f.cpu().numpy() - r["forces"]) ** 2)) * HARTREE_TO_KCALMOL
        assert rmse <= tol_f
    return e, f


@pytest.mark.parametrize("which", ["pot", "pot_tc"])
def test_isolated_atoms_and_small_systems(which, request):
    p = request.getfixturevalue(which)
    rng = np.random.default_rng(0)
    iso = rng.uniform(-1, 1, (5, 3)) * 50.0          # five atoms far apart: empty rows
    pair = np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 6.0]])  # beyond 5.2 A
    one = np.zeros((1, 3))
    mol = molecule_batch(1, seed=2)[0]
    xyz = np.concatenate([iso, pair, one, mol.coordinates])
    sp = np.concatenate([[1, 6, 7, 8, 17], [8, 8], [16], mol.species])
    nat = [5, 2, 1, mol.natoms]
    e, f = check(p, xyz, sp, nat)
    np.testing.assert_allclose(f.cpu().numpy()[:8], 0.0, atol=1e-7)


def test_empty_system_inside_a_batch(pot):
    mols = molecule_batch(2, seed=5)
    xyz = np.concatenate([m.coordinates for m in mols])
    sp = np.concatenate([m.species for m in mols])
    e, f = pot.energy_and_forces(xyz, sp, [mols[0].natoms, 0, mols[1].natoms])
    e_ref, f_ref = pot.energy_and_forces(xyz, sp, [mols[0].natoms, mols[1].natoms])
    e, e_ref = e.cpu().numpy(), e_ref.cpu().numpy()
    assert e.shape == (3,) and e[1] == 0.0
    np.testing.assert_allclose(e[[0, 2]], e_ref, rtol=0, atol=1e-9)


def test_empty_batch(pot):
    e, f = pot.energy_and_forces(np.zeros((0, 3)), np.zeros(0, np.int64), [0])
    assert tuple(f.shape) == (0, 3) and tuple(e.shape) == (1,) and float(e.abs().sum()) == 0.0


def test_one_species_only(pot_tc):
    """Only carbon atoms: a single tile species, six networks unused."""
    mol = molecule_batch(1, seed=9, nmin=30, nmax=30)[0]
    check(pot_tc, mol.coordinates, np.full(mol.natoms, 6), [mol.natoms])


@pytest.mark.parametrize("elements", [(1, 6, 8), (6,)])
def test_more_than_96_angular_neighbours(cuda_device, elements):
    """120 atoms inside a 1.7 A sphere: every atom has 119 angular neighbours
    (the staging follows the row capacity, regrown from the first guess),
    three species or one (a single 119-neighbour block), against the FP64
    oracle."""
    from fennol_b200.params import AEVConfig, MLPConfig
    from fennol_b200.potential import ANIPotential, HARTREE_TO_KCALMOL
    from oracle import ani_ref

    rng = np.random.default_rng(5)
    pts = []
    while len(pts) < 120:
        p = rng.uniform(-1.7, 1.7, 3)
        if np.linalg.norm(p) < 1.7 and all(np.linalg.norm(p - q) > 0.15 for q in pts):
            pts.append(p)
    xyz = np.array(pts)
    sp = rng.choice(list(elements), size=120)
    pot = ANIPotential(precision="fp32", device=cuda_device, seed=0)
    e, f = pot.energy_and_forces(xyz, sp, [120])
    layout, g, ws = next(iter(pot._cache.values()))
    assert g.cap_r >= 119
    r = ani_ref.energy_and_forces(xyz, sp, [120], pot.weights, AEVConfig(), MLPConfig())
    de = abs(float(e[0]) - r["energy"][0]) * HARTREE_TO_KCALMOL / 120
    scale = np.abs(r["forces"]).max()
    # atomic energies reach 1e4 kcal/mol in so dense a cluster: float32 rounding, relative
    e_atom = abs(r["energy"][0]) * HARTREE_TO_KCALMOL / 120
    assert de < 2e-6 * e_atom + 1e-4, (de, e_atom)
    np.testing.assert_allclose(f.cpu().numpy(), r["forces"], rtol=0, atol=1e-4 * scale)
