"""Size-independent parity at large sizes: a k x k x k supercell of a periodic
box has every atom in the same environment as in the box, so its energy is
k^3 times the box's and each copy carries the box's forces.  Checked for
98,304 and 331,776 atoms, and for the BF16 form with an 8-model ensemble.

The copies sit up to 150 A from the origin, where float32 positions are
~10x coarser than in the box, so the comparison allows float32 position
rounding: 1e-5 kcal/mol/atom in energy, 1e-4 of the largest force."""

import numpy as np
import pytest

from fennol_b200.potential import ANIPotential, HARTREE_TO_KCALMOL
from fennol_b200.systems import water_box

pytestmark = pytest.mark.gpu


def supercell(s, k):
    L = s.cell[0, 0]
    shifts = np.array([[a, b, c] for a in range(k) for b in range(k) for c in range(k)], dtype=np.float64) * L
    xyz = (s.coordinates[None, :, :] + shifts[:, None, :]).reshape(-1, 3)
    return xyz, np.tile(s.species, k ** 3), s.cell * k


@pytest.mark.parametrize("k,precision,models", [(2, "fp32", 1), (3, "bf16x2", 1), (2, "bf16x2", 8)])
def test_supercell_energy_and_forces(cuda_device, k, precision, models):
    s = water_box(16, seed=11)  # 12,288 atoms, 49.7 A
    pot = ANIPotential(precision=precision, bf16_weights=precision != "fp32", n_models=models,
                       device=cuda_device, seed=0)
    e1, f1 = pot.energy_and_forces(s.coordinates, s.species, [s.natoms], s.cell[None])
    e1, f1 = float(e1[0]), f1.cpu().numpy().copy()
    xyz, sp, cell = supercell(s, k)
    ek, fk = pot.energy_and_forces(xyz, sp, [xyz.shape[0]], cell[None])
    ek, fk = float(ek[0]), fk.cpu().numpy().reshape(k ** 3, s.natoms, 3)
    n = xyz.shape[0]
    assert abs(ek - k ** 3 * e1) * HARTREE_TO_KCALMOL / n <= 1e-5
    scale = np.abs(f1).max()
    for c in range(k ** 3):
        np.testing.assert_allclose(fk[c], f1, rtol=0, atol=1e-4 * scale)
