"""Model hyper-parameters and weights of the ANI-2x-style potential.

The hyper-parameter names follow FeNNol's ``ANIAEV`` module
(``src/fennol/models/embeddings/ani.py:18-44``) and the per-species network
of ``SpeciesIndexNet`` (``src/fennol/models/misc/nets.py:301-350``).  Weights
are stored exactly like a Flax ``Dense`` layer: ``kernel[in, out]`` and
``bias[out]`` with ``y = x @ kernel + bias``; one network per species, layers
named ``Layer_1 .. Layer_4`` (``nets.py:82-98``).
"""

from __future__ import annotations

import dataclasses
from typing import Dict, List, Sequence, Tuple

import numpy as np

# Chemical symbols by atomic number (only the light elements the ANI family uses
# are needed on this path; index = atomic number).
PERIODIC_TABLE = [
    "Dummy", "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne",
    "Na", "Mg", "Al", "Si", "P", "S", "Cl", "Ar", "K", "Ca",
]
PERIODIC_TABLE_REV_IDX = {s: i for i, s in enumerate(PERIODIC_TABLE)}

# Standard atomic weights (Da) used by the MD integrator; same values as
# ``src/fennol/utils/periodic_table.py`` ATOMIC_MASSES for these elements.
ATOMIC_MASSES = {
    1: 1.008, 6: 12.011, 7: 14.007, 8: 15.999, 9: 18.99840316,
    15: 30.973762, 16: 32.06, 17: 35.45,
}



def atomic_masses(species) -> np.ndarray:
    """Masses (Da, float64) of an array of atomic numbers; unknown elements raise."""
    z = np.asarray(species, dtype=np.int64)
    table = _MASS_TABLE[np.clip(z, 0, _MASS_TABLE.shape[0] - 1)]
    if z.size and (z.min() < 0 or z.max() >= _MASS_TABLE.shape[0] or np.any(table == 0)):
        raise ValueError("atomic number without a mass in ATOMIC_MASSES")
    return table


_MASS_TABLE = np.zeros(max(ATOMIC_MASSES) + 1)
for _z, _m in ATOMIC_MASSES.items():
    _MASS_TABLE[_z] = _m

ANI2X_SPECIES = ("H", "C", "N", "O", "S", "F", "Cl")

# Last-layer scale of the random model used by MD workloads (see init_weights).
MD_OUTPUT_SCALE = 0.02


@dataclasses.dataclass(frozen=True)
class AEVConfig:
    """ANIAEV hyper-parameters (``ani.py:18-44``).

    Defaults are the ANI-2x set used by the water-box and molecule workloads:
    radial 16 shifts 0.9-5.2 A (eta 19.7), angular 4 sections x 8 shifts
    0.9-3.5 A (eta 12.5, zeta 14.1).  Output width
    ``S*radial_dist_divisions + S(S+1)/2*angle_sections*angular_dist_divisions``
    = 1008 for 7 species.
    """

    species_order: Tuple[str, ...] = ANI2X_SPECIES
    radial_cutoff: float = 5.2
    angular_cutoff: float = 3.5
    radial_eta: float = 19.7
    angular_eta: float = 12.5
    radial_dist_divisions: int = 16
    angular_dist_divisions: int = 8
    zeta: float = 14.1
    angle_sections: int = 4
    radial_start: float = 0.9
    angular_start: float = 0.9

    @property
    def num_species(self) -> int:
        return len(self.species_order)

    @property
    def num_species_pair(self) -> int:
        s = self.num_species
        return s * (s + 1) // 2

    @property
    def radial_length(self) -> int:
        return self.num_species * self.radial_dist_divisions

    @property
    def angular_sublength(self) -> int:
        return self.angle_sections * self.angular_dist_divisions

    @property
    def aev_length(self) -> int:
        return self.radial_length + self.num_species_pair * self.angular_sublength

    def radial_shifts(self) -> np.ndarray:
        """``linspace(radial_start, cutoff, RD+1)[:-1]`` (ani.py:73-78)."""
        return np.linspace(self.radial_start, self.radial_cutoff,
                           self.radial_dist_divisions + 1)[:-1]

    def angular_shifts(self) -> np.ndarray:
        """``linspace(angular_start, angular_cutoff, AD+1)[:-1]`` (ani.py:104-109)."""
        return np.linspace(self.angular_start, self.angular_cutoff,
                           self.angular_dist_divisions + 1)[:-1]

    def angle_shifts(self) -> np.ndarray:
        """``linspace(0, pi, AS+1)[:-1] + pi/(2 AS)`` (ani.py:99-103)."""
        return (np.linspace(0, np.pi, self.angle_sections + 1)
                + np.pi / (2 * self.angle_sections))[:-1]

    def species_index(self, atomic_numbers: np.ndarray) -> np.ndarray:
        """Map atomic numbers to positions in ``species_order`` (ani.py:49-60).

        Raises ``ValueError`` for an element the model does not handle, like
        ``SpeciesIndexNet`` with ``check_unhandled`` (nets.py:392-395).
        """
        conv = np.full(len(PERIODIC_TABLE), -1, dtype=np.int32)
        for k, sym in enumerate(self.species_order):
            conv[PERIODIC_TABLE_REV_IDX[sym]] = k
        z = np.asarray(atomic_numbers, dtype=np.int64)
        if z.size and (z.min() < 0 or z.max() >= conv.shape[0]):
            raise ValueError("atomic number outside the supported table")
        idx = conv[z]
        if z.size and idx.min() < 0:
            bad = sorted(set(int(v) for v in z[idx < 0]))
            raise ValueError(f"species {bad} not handled by this model "
                             f"(handled: {self.species_order})")
        return idx.astype(np.int32)


@dataclasses.dataclass(frozen=True)
class MLPConfig:
    """Per-species FullyConnectedNet (``nets.py:13-102``): CELU(alpha) hidden layers."""

    hidden: Tuple[int, ...] = (256, 192, 160)
    output_dim: int = 1
    celu_alpha: float = 0.1


# weights[model][species_symbol] = [(kernel[in,out], bias[out]), ...] (float64)
Weights = List[Dict[str, List[Tuple[np.ndarray, np.ndarray]]]]


def init_weights(aev: AEVConfig, mlp: MLPConfig, seed: int = 0,
                 n_models: int = 1, bias_std: float = 0.0, output_scale: float = 1.0) -> Weights:
    """Seeded random weights: kernel ~ N(0, 1/fan_in), bias 0 (or N(0, bias_std)).

    Model ``m`` of an ensemble uses seed ``seed + 1000*m`` so that members are
    independent.  ``output_scale`` multiplies the last layer's kernel: with
    the unscaled N(0, 1/fan_in) network atomic energies vary by ~40 kcal/mol
    and the random landscape pulls atoms together within ~10 fs of MD, so MD
    workloads use a small scale (0.02) that keeps forces near thermal size.
    Float64 master copy; device packing casts as needed.
    """
    dims = [aev.aev_length, *mlp.hidden, mlp.output_dim]
    out: Weights = []
    for m in range(n_models):
        rng = np.random.default_rng(seed + 1000 * m)
        model = {}
        for sym in aev.species_order:
            layers = []
            for din, dout in zip(dims[:-1], dims[1:]):
                w = rng.standard_normal((din, dout)) / np.sqrt(din)
                if dout == dims[-1] and din == dims[-2]:
                    w = w * output_scale
                if bias_std > 0:
                    b = rng.standard_normal(dout) * bias_std
                else:
                    b = np.zeros(dout)
                layers.append((w, b))
            model[sym] = layers
        out.append(model)
    return out


def weights_to_variables(weights: Weights, module_name: str = "energy") -> List[dict]:
    """Express weights as FeNNol ``variables`` trees, one per model:
    ``{"params": {module_name: {sym: {"Layer_k": {"kernel", "bias"}}}}}``
    (the layout ``FENNIX.save`` serialises, ``fennix.py:635-662``)."""
    trees = []
    for model in weights:
        p = {}
        for sym, layers in model.items():
            p[sym] = {f"Layer_{k + 1}": {"kernel": np.asarray(w), "bias": np.asarray(b)}
                      for k, (w, b) in enumerate(layers)}
        trees.append({"params": {module_name: p}})
    return trees


def variables_to_weights(trees: Sequence[dict], species_order: Sequence[str],
                         module_name: str = "energy") -> Weights:
    """Inverse of :func:`weights_to_variables` (reads a FeNNol variables tree)."""
    out: Weights = []
    for tree in trees:
        p = tree["params"][module_name]
        model = {}
        for sym in species_order:
            net = p[sym]
            nl = len([k for k in net if k.startswith("Layer_")])
            model[sym] = [(np.asarray(net[f"Layer_{k + 1}"]["kernel"], dtype=np.float64),
                           np.asarray(net[f"Layer_{k + 1}"]["bias"], dtype=np.float64))
                          for k in range(nl)]
        out.append(model)
    return out
