"""The ASE calculator's protocol on the CPU: unit conversion to eV, Voigt
stress, recomputation only when the atoms change, and FeNNol's PBC rule.
A harmonic stand-in model replaces the CUDA potential."""

import numpy as np
import pytest
import torch

from fennol_b200.ase_calculator import FENNIXCalculator, _voigt
from fennol_b200.fennix import energy_multiplier

EV = energy_multiplier("eV")


class Atoms:
    """The ase.Atoms accessors the calculator reads."""

    def __init__(self, numbers, positions, cell=None, pbc=False):
        self.numbers = np.asarray(numbers)
        self.positions = np.asarray(positions, dtype=np.float64)
        self.cell = np.zeros((3, 3)) if cell is None else np.asarray(cell, dtype=np.float64)
        self.pbc = np.array([pbc] * 3 if np.isscalar(pbc) else pbc, dtype=bool)

    def get_positions(self):
        return self.positions.copy()

    def get_atomic_numbers(self):
        return self.numbers.copy()

    def get_cell(self, complete=False):
        return self.cell.copy()

    def get_pbc(self):
        return self.pbc.copy()

    def get_volume(self):
        return abs(np.linalg.det(self.cell))


class Harmonic:
    """E = 0.5 k sum x^2 in kcal/mol (a model unit other than Ha), virial = S."""

    Ha_to_model_energy = energy_multiplier("kcalpermol")

    def __init__(self):
        self.calls = 0
        self.vir = np.array([[1.0, 0.2, 0.0], [0.4, 2.0, 0.0], [0.0, 0.0, 3.0]])

    def _ef(self, coordinates):
        self.calls += 1
        x = torch.tensor(coordinates, dtype=torch.float64)
        return (0.5 * (x ** 2).sum()).reshape(1), -x

    def total_energy(self, gpu_preprocessing=False, **inputs):
        e, _ = self._ef(inputs["coordinates"])
        return e, {}

    def energy_and_forces(self, gpu_preprocessing=False, **inputs):
        e, f = self._ef(inputs["coordinates"])
        return e, f, {}

    def energy_and_forces_and_virial(self, gpu_preprocessing=False, **inputs):
        e, f = self._ef(inputs["coordinates"])
        return e, f, torch.tensor(self.vir)[None], {}

    def set_energy_terms(self, terms, jit=True):
        self.terms = terms


def test_units_forces_and_caching():
    m = Harmonic()
    calc = FENNIXCalculator(m, energy_terms=["energy"])
    assert m.terms == ["energy"]
    a = Atoms([8, 1, 1], [[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 2.0, 0.0]])
    conv = EV / energy_multiplier("kcalpermol")
    assert calc.get_potential_energy(a) == pytest.approx(0.5 * 5.0 * conv)
    assert m.calls == 1
    assert calc.get_potential_energy(a) == pytest.approx(0.5 * 5.0 * conv)
    assert m.calls == 1                                  # unchanged atoms: no new evaluation
    np.testing.assert_allclose(calc.get_forces(a), -a.positions * conv)
    a.positions[1, 0] = 2.0
    assert calc.get_potential_energy(a) == pytest.approx(0.5 * 8.0 * conv)


def test_stress_is_the_virial_over_the_volume_in_voigt_order():
    m = Harmonic()
    calc = FENNIXCalculator(m)
    a = Atoms([8], [[0.1, 0.2, 0.3]], cell=np.diag([10.0, 11.0, 12.0]), pbc=True)
    s = calc.get_stress(a)
    conv = EV / energy_multiplier("kcalpermol")
    np.testing.assert_allclose(s, _voigt(m.vir) * conv / 1320.0)
    assert s[5] == pytest.approx(0.3 * conv / 1320.0)     # symmetrised xy


def test_partial_pbc_is_rejected():
    calc = FENNIXCalculator(Harmonic())
    a = Atoms([8], [[0.0, 0.0, 0.0]], cell=np.eye(3) * 10, pbc=[True, True, False])
    with pytest.raises(NotImplementedError):
        calc.get_potential_energy(a)
