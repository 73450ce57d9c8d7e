"""GPU parity of the AEV, energies and forces against the FP64 oracle.

Tolerances (from the error budget of the path): force RMSE <= 0.05
kcal/mol/A and |dE|/N <= 1e-4 kcal/mol/atom against the FP64 oracle;
AEV features within 2e-5 absolute + 1e-4 relative (float32 kernel)."""

from pathlib import Path

import numpy as np
import pytest
import torch

from fennol_b200.params import AEVConfig, MLPConfig, init_weights
from fennol_b200.potential import ANIPotential, HARTREE_TO_KCALMOL
from fennol_b200.systems import molecule_batch, water_box
from oracle import ani_ref

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).parent / "golden"
CFG, MCFG = AEVConfig(), MLPConfig()
FORCE_RMSE_TOL = 0.05   # kcal/mol/A
ENERGY_TOL = 1e-4       # kcal/mol/atom


def errors(e, f, ref_e, ref_f, natoms):
    de = np.abs(np.asarray(e) - ref_e) * HARTREE_TO_KCALMOL / np.asarray(natoms)
    rmse = np.sqrt(np.mean((np.asarray(f) - ref_f) ** 2)) * HARTREE_TO_KCALMOL
    return float(de.max()), float(rmse)


@pytest.fixture(scope="module")
def pot32(cuda_device):
    return ANIPotential(precision="fp32", device=cuda_device, seed=0)


def test_golden_water64_energy_forces(pot32):
    d = np.load(GOLDEN / "water64.npz")
    e, f = pot32.energy_and_forces(d["coordinates"], d["species"], [192], d["cell"][None])
    de, rmse = errors(e.cpu().numpy(), f.cpu().numpy(), d["energy"], d["forces"], [192])
    assert de <= ENERGY_TOL and rmse <= FORCE_RMSE_TOL, (de, rmse)
    # much tighter in practice for the float32 form
    assert rmse < 5e-3


def test_aev_rows_match_oracle(pot32, cuda_device):
    d = np.load(GOLDEN / "water64.npz")
    pot32.energy_and_forces(d["coordinates"], d["species"], [192], d["cell"][None])
    layout, g, ws = next(iter(pot32._cache.values()))
    rows = ws.x.float().cpu().numpy()[layout.atom_row_host[:8], :1008]
    np.testing.assert_allclose(rows, d["aev_rows"], rtol=1e-4, atol=2e-5)


def test_golden_molecules(pot32):
    d = np.load(GOLDEN / "molecules6.npz")
    e, f = pot32.energy_and_forces(d["coordinates"], d["species"], d["natoms"])
    de, rmse = errors(e.cpu().numpy(), f.cpu().numpy(), d["energy"], d["forces"], d["natoms"])
    assert de <= ENERGY_TOL and rmse <= FORCE_RMSE_TOL, (de, rmse)


@pytest.mark.parametrize("n_side,seed", [(8, 1), (12, 2)])
def test_water_boxes_vs_fp64(pot32, n_side, seed):
    s = water_box(n_side, seed=seed)
    r = ani_ref.energy_and_forces(s.coordinates, s.species, [s.natoms], pot32.weights, CFG, MCFG,
                                  cells=s.cell[None])
    e, f = pot32.energy_and_forces(s.coordinates, s.species, [s.natoms], s.cell[None])
    de, rmse = errors(e.cpu().numpy(), f.cpu().numpy(), r["energy"], r["forces"], [s.natoms])
    assert de <= ENERGY_TOL and rmse <= FORCE_RMSE_TOL, (de, rmse)


def test_net_force_vanishes(pot32):
    s = water_box(8, seed=3)
    _, f = pot32.energy_and_forces(s.coordinates, s.species, [s.natoms], s.cell[None])
    net = f.double().sum(0).cpu().numpy() * HARTREE_TO_KCALMOL
    assert np.abs(net).max() < 1e-2


def test_ensemble_mean(cuda_device):
    W = init_weights(CFG, MCFG, seed=7, n_models=3)
    pot = ANIPotential(precision="fp32", device=cuda_device, weights=W)
    mols = molecule_batch(5, seed=12)
    xyz = np.concatenate([m.coordinates for m in mols])
    sp = np.concatenate([m.species for m in mols])
    nat = [m.natoms for m in mols]
    r = ani_ref.energy_and_forces(xyz, sp, nat, W, CFG, MCFG)
    e, f = pot.energy_and_forces(xyz, sp, nat)
    de, rmse = errors(e.cpu().numpy(), f.cpu().numpy(), r["energy"], r["forces"], nat)
    assert de <= ENERGY_TOL and rmse <= FORCE_RMSE_TOL, (de, rmse)


def test_batched_equals_alone(pot32):
    """Each system's result is the same alone and inside a mixed batch."""
    box = water_box(6, seed=4)
    mols = molecule_batch(4, seed=13)
    systems = [mols[0], box, mols[1], mols[2], mols[3]]
    cells = [None, box.cell, None, None, None]
    xyz = np.concatenate([s.coordinates for s in systems])
    sp = np.concatenate([s.species for s in systems])
    nat = [s.natoms for s in systems]
    e_mix, f_mix = pot32.energy_and_forces(xyz, sp, nat, cells)
    e_mix, f_mix = e_mix.cpu().numpy().copy(), f_mix.cpu().numpy().copy()
    off = np.concatenate([[0], np.cumsum(nat)])
    for b, s in enumerate(systems):
        c = None if cells[b] is None else cells[b][None]
        e, f = pot32.energy_and_forces(s.coordinates, s.species, [s.natoms], c)
        assert abs(float(e[0]) - e_mix[b]) * HARTREE_TO_KCALMOL / s.natoms < 1e-6
        np.testing.assert_allclose(f.cpu().numpy(), f_mix[off[b]:off[b + 1]], atol=2e-5)


def test_staged_adjoint_matches_unstaged(cuda_device):
    """fennol_aev_backward_staged (reading the staging saved by
    fennol_aev_forward_staged) gives the forces of fennol_aev_backward, and
    the staged forward writes the same AEV rows as the plain one."""
    from fennol_b200 import _lib
    from fennol_b200._lib import call
    from fennol_b200.potential import C_ptr, _ptr

    pot = ANIPotential(precision="bf16x2", device=cuda_device, seed=0, bf16_weights=True)
    s = water_box(6, seed=31)
    x = torch.tensor(s.coordinates, dtype=torch.float32, device=cuda_device)
    pot.energy_and_forces(x, s.species, [s.natoms], s.cell[None])
    lay, g, ws = next(iter(pot._cache.values()))
    st = torch.cuda.current_stream().cuda_stream
    lp = C_ptr(pot.params)
    args = (ws.xyzs.data_ptr(), lay.n, lay.t_atom_sys.data_ptr(), lay.t_cell.data_ptr(), g.rad_j.data_ptr(),
            g.rad_s.data_ptr(), g.rad_n.data_ptr(), g.cap_r, lp, lay.t_atom_row.data_ptr())
    rows = lay.t_atom_row.long()
    call("fennol_aev_forward", *args, ws.aev_kind, ws.x.data_ptr(), _ptr(ws.x_lo), ws.x.shape[1],
         ws.status.data_ptr(), st)
    x_plain = ws.x[rows].clone()
    call("fennol_aev_forward_staged", *args, ws.aev_kind, ws.x.data_ptr(), _ptr(ws.x_lo), ws.x.shape[1],
         g.aev_stage.data_ptr(), g.aev_stage.numel(), ws.status.data_ptr(), st)
    assert torch.equal(ws.x[rows], x_plain)
    ws.dx.normal_()  # any dE/dAEV rows
    f = []
    for name, extra in (("fennol_aev_backward", ()), ("fennol_aev_backward_staged", (g.aev_stage.data_ptr(),))):
        ws.forces4.zero_()
        call(name, *args, ws.dx.data_ptr(), ws.dx.shape[1], ws.forces4.data_ptr(), *extra,
             ws.status.data_ptr(), st)
        f.append(ws.forces4[:lay.n, :3].cpu().numpy().copy())
    assert int(ws.status[_lib.ST_ANG_OVERFLOW]) == 0
    scale = np.abs(f[0]).max()
    np.testing.assert_allclose(f[1], f[0], atol=1e-5 * scale, rtol=0)
