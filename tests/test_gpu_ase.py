"""The ASE calculator on the CUDA path: energy, forces and stress in eV and
Angstrom equal the FENNIX model's own outputs converted from Hartree."""

import numpy as np
import pytest

from fennol_b200.ase_calculator import FENNIXCalculator, _voigt
from fennol_b200.fennix import energy_multiplier
from fennol_b200.systems import water_box
from test_ase_calculator import Atoms
from test_gpu_fennix import make_model

pytestmark = pytest.mark.gpu


def test_calculator_matches_the_model(cuda_device):
    m = make_model(rng_key=0)
    s = water_box(4, seed=51)
    a = Atoms(s.species, s.coordinates, cell=np.asarray(s.cell).reshape(3, 3), pbc=True)
    calc = FENNIXCalculator(m)
    e_ev = calc.get_potential_energy(a)
    f_ev = calc.get_forces(a)
    stress = calc.get_stress(a)
    cell = np.asarray(s.cell).reshape(3, 3)
    e, f, vir, _ = m.energy_and_forces_and_virial(
        species=np.asarray(s.species), coordinates=np.asarray(s.coordinates, dtype=np.float32),
        natoms=np.array([s.natoms]), cells=cell[None], reciprocal_cells=np.linalg.inv(cell)[None])
    ev = energy_multiplier("eV")
    assert e_ev == pytest.approx(float(e[0]) * ev, rel=1e-9)
    scale = np.abs(f.cpu().numpy()).max() * ev
    np.testing.assert_allclose(f_ev, f.cpu().numpy() * ev, atol=1e-5 * scale)
    vol = abs(np.linalg.det(cell))
    np.testing.assert_allclose(stress, _voigt(vir[0].cpu().numpy()) * ev / vol,
                               atol=1e-5 * np.abs(stress).max())
    # a move recomputes
    a.positions[0, 0] += 0.05
    assert calc.get_potential_energy(a) != e_ev
