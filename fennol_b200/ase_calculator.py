"""ASE calculator over the CUDA energy path: FeNNol's ``FENNIXCalculator``
(``src/fennol/ase.py:13-200``) with the same constructor arguments, the
properties ``energy``, ``forces`` and ``stress`` in eV and Angstrom, and the
same input rules (periodic in all three directions or in none).

With ASE installed the class is an ``ase.calculators.calculator.Calculator``
and plugs into ASE's optimisers and MD.  Without ASE (as in this image) the
same class works on any object with the ``ase.Atoms`` accessors it reads
(``get_positions``, ``get_atomic_numbers``, ``get_cell``, ``get_pbc``,
``get_volume``) through ``get_potential_energy``, ``get_forces`` and
``get_stress``, recomputing when positions, numbers or the cell change.
"""

from __future__ import annotations

import os
from typing import Optional, Sequence, Union

import numpy as np

from .fennix import FENNIX, energy_multiplier

try:  # pragma: no cover - depends on the environment
    from ase.calculators.calculator import Calculator as _Base
    from ase.calculators.calculator import all_changes
    HAVE_ASE = True
except ImportError:
    HAVE_ASE = False
    all_changes = ["positions", "numbers", "cell", "pbc", "initial_charges", "initial_magmoms"]

    class _Base:
        """The part of ASE's Calculator protocol this calculator uses."""

        implemented_properties: Sequence[str] = ()

        def __init__(self, **kwargs):
            self.atoms = None
            self.results = {}
            self._state = None

        @staticmethod
        def _snapshot(atoms):
            return (np.array(atoms.get_positions(), dtype=np.float64),
                    np.array(atoms.get_atomic_numbers()),
                    np.array(_cell_array(atoms), dtype=np.float64),
                    np.array(atoms.get_pbc(), dtype=bool))

        def calculate(self, atoms=None, properties=("energy",), system_changes=all_changes):
            if atoms is not None:
                self.atoms = atoms
                self._state = self._snapshot(atoms)

        def _changes(self, atoms):
            if self._state is None:
                return list(all_changes)
            new = self._snapshot(atoms)
            names = ("positions", "numbers", "cell", "pbc")
            return [n for n, a, b in zip(names, self._state, new)
                    if a.shape != b.shape or not np.array_equal(a, b)]

        def get_property(self, name, atoms=None, allow_calculation=True):
            atoms = self.atoms if atoms is None else atoms
            changes = self._changes(atoms)
            if changes:
                self.results = {}
            if name not in self.results:
                if not allow_calculation:
                    return None
                self.calculate(atoms, [name], changes or list(all_changes))
            return self.results[name]

        def get_potential_energy(self, atoms=None, force_consistent=False):
            return self.get_property("energy", atoms)

        def get_forces(self, atoms=None):
            return self.get_property("forces", atoms).copy()

        def get_stress(self, atoms=None):
            return self.get_property("stress", atoms).copy()


def _cell_array(atoms) -> np.ndarray:
    cell = atoms.get_cell()
    try:
        cell = atoms.get_cell(complete=True)
    except TypeError:
        pass
    return np.asarray(getattr(cell, "array", cell), dtype=np.float64).reshape(3, 3)


def _voigt(stress: np.ndarray) -> np.ndarray:
    """3 x 3 -> (xx, yy, zz, yz, xz, xy), symmetrised."""
    s = 0.5 * (stress + stress.T)
    return np.array([s[0, 0], s[1, 1], s[2, 2], s[1, 2], s[0, 2], s[0, 1]])


class FENNIXCalculator(_Base):
    """FENNIX calculator for ASE on the CUDA path.

    ``model``: a FENNIX model or the path of a ``.fnx`` / ``.pkl`` file.
    ``use_float64``: accepted; the CUDA path computes the network in its own
    precision (energies are reduced in float64).  ``matmul_prec``:
    ``"highest"`` selects the FP32 network form when loading from a file,
    ``"default"`` / ``"high"`` the split-BF16 tensor-core form.
    ``gpu_preprocessing``: the fixed-capacity preprocessing path (lists are
    built on the GPU either way).  ``energy_terms``: see
    ``FENNIX.set_energy_terms``.  ``save_raw_output``: keep the model output
    in ``results["raw_output"]``.
    """

    implemented_properties = ["energy", "forces", "stress"]

    def __init__(self, model: Union[str, FENNIX], gpu_preprocessing: bool = False, atoms=None,
                 verbose: bool = False, energy_terms: Optional[Sequence[str]] = None,
                 use_float64: bool = False, matmul_prec: Optional[str] = None,
                 save_raw_output: bool = False, **kwargs):
        super().__init__()
        if matmul_prec is not None and matmul_prec not in ("default", "high", "highest"):
            raise ValueError("matmul_prec should be one of 'default', 'high', 'highest'")
        if not isinstance(model, (str, bytes, os.PathLike)):
            self.model = model  # a FENNIX model (or an object with its methods)
        else:
            if matmul_prec is not None and "precision" not in kwargs:
                kwargs["precision"] = "fp32" if matmul_prec == "highest" else "bf16x2"
            self.model = FENNIX.load(model, **kwargs)
        if energy_terms is not None:
            self.model.set_energy_terms(energy_terms)
        self.dtype = "float64" if use_float64 else "float32"
        self.gpu_preprocessing = gpu_preprocessing
        self.verbose = verbose
        self.save_raw_output = save_raw_output
        # model output -> eV, as the reference's ase.units.Hartree / model unit
        self.energy_conv = energy_multiplier("eV") / self.model.Ha_to_model_energy
        if atoms is not None:
            self.atoms = atoms

    def _inputs(self, atoms):
        pbc = np.asarray(atoms.get_pbc(), dtype=bool).reshape(-1)
        if pbc.any() and not pbc.all():
            raise NotImplementedError("PBC should be activated in all directions.")
        species = np.asarray(atoms.get_atomic_numbers(), dtype=np.int32)
        inputs = {"species": species,
                  "coordinates": np.asarray(atoms.get_positions(), dtype=self.dtype),
                  "natoms": np.array([species.shape[0]], dtype=np.int32),
                  "batch_index": np.zeros(species.shape[0], dtype=np.int32)}
        if pbc.all():
            cell = _cell_array(atoms)
            inputs["cells"] = cell.reshape(1, 3, 3)
            inputs["reciprocal_cells"] = np.linalg.inv(cell).reshape(1, 3, 3)
        return inputs

    def calculate(self, atoms=None, properties=("energy",), system_changes=all_changes):
        super().calculate(atoms, properties, system_changes)
        inputs = self._inputs(self.atoms)
        results = {}
        if "stress" in properties:
            e, f, virial, output = self.model.energy_and_forces_and_virial(
                gpu_preprocessing=self.gpu_preprocessing, **inputs)
            volume = float(self.atoms.get_volume())
            stress = np.asarray(virial[0].detach().cpu().numpy(), dtype=np.float64) * self.energy_conv / volume
            results["stress"] = _voigt(stress)
            results["forces"] = np.asarray(f.detach().cpu().numpy(), dtype=np.float64) * self.energy_conv
        elif "forces" in properties:
            e, f, output = self.model.energy_and_forces(gpu_preprocessing=self.gpu_preprocessing, **inputs)
            results["forces"] = np.asarray(f.detach().cpu().numpy(), dtype=np.float64) * self.energy_conv
        else:
            e, output = self.model.total_energy(gpu_preprocessing=self.gpu_preprocessing, **inputs)
        results["energy"] = float(e[0]) * self.energy_conv
        if self.save_raw_output:
            results["raw_output"] = output
        self.results.update(results)
