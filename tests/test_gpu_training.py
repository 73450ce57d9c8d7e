"""Training-loss parameter gradients through the hand-written adjoints
(AEV tangent kernel + explicit network sweep) against second-order autograd
of the FP64 oracle and against finite differences of the FP64 loss."""

import numpy as np
import pytest
import torch

from fennol_b200.params import AEVConfig, MLPConfig, init_weights
from fennol_b200.potential import ANIPotential
from fennol_b200.systems import molecule_batch, water_box
from fennol_b200.training import LossGradient, flatten
from oracle import ani_ref

pytestmark = pytest.mark.gpu
CFG, MCFG = AEVConfig(), MLPConfig()
REL_TOL = 2e-4  # relative L2 error of the whole gradient vector against FP64


def batch(n_mol, seed):
    mols = molecule_batch(n_mol, seed=seed)
    xyz = np.concatenate([m.coordinates for m in mols])
    sp = np.concatenate([m.species for m in mols])
    return xyz, sp, np.array([m.natoms for m in mols])


def teacher_targets(xyz, sp, nat, cells=None):
    teacher = init_weights(CFG, MCFG, seed=77)
    r = ani_ref.energy_and_forces(xyz, sp, nat, teacher, CFG, MCFG, cells=cells)
    return r["energy"], r["forces"]


def rel_err(g, g_ref):
    a, b = flatten(g, CFG.species_order), flatten(g_ref, CFG.species_order)
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_gradient_matches_second_order_autograd(cuda_device, dtype):
    xyz, sp, nat = batch(24, seed=41)
    W = init_weights(CFG, MCFG, seed=5, bias_std=0.05)
    e_ref, f_ref = teacher_targets(xyz, sp, nat)
    pot = ANIPotential(precision="fp32", device=cuda_device, weights=W)
    terms, g = LossGradient(pot, w_e=1.0, w_f=10.0, dtype=dtype)(xyz, sp, nat, e_ref, f_ref)
    loss_ref, g_ref = ani_ref.loss_and_grads(xyz, sp, nat, W[0], CFG, MCFG, e_ref, f_ref)
    assert abs(terms.loss - loss_ref) <= 1e-4 * loss_ref
    assert rel_err(g, g_ref) < REL_TOL
    for sym in CFG.species_order:
        for (gw, gb), (rw, rb) in zip(g[sym], g_ref[sym]):
            scale = max(np.abs(rw).max(), 1e-30)
            np.testing.assert_allclose(gw, rw, rtol=0, atol=2e-3 * scale)


def test_force_term_alone_and_energy_term_alone(cuda_device):
    """Each seed path on its own (w_e = 0 exercises the tangent kernel only)."""
    xyz, sp, nat = batch(12, seed=43)
    W = init_weights(CFG, MCFG, seed=6, bias_std=0.05)
    e_ref, f_ref = teacher_targets(xyz, sp, nat)
    pot = ANIPotential(precision="fp32", device=cuda_device, weights=W)
    for w_e, w_f in ((0.0, 1.0), (1.0, 0.0)):
        _, g = LossGradient(pot, w_e=w_e, w_f=w_f)(xyz, sp, nat, e_ref, f_ref)
        _, g_ref = ani_ref.loss_and_grads(xyz, sp, nat, W[0], CFG, MCFG, e_ref, f_ref, w_e=w_e, w_f=w_f)
        assert rel_err(g, g_ref) < REL_TOL, (w_e, w_f)


def test_periodic_box_gradient(cuda_device):
    s = water_box(4, seed=12)
    W = init_weights(CFG, MCFG, seed=8, bias_std=0.05)
    e_ref, f_ref = teacher_targets(s.coordinates, s.species, [s.natoms], s.cell[None])
    pot = ANIPotential(precision="fp32", device=cuda_device, weights=W)
    _, g = LossGradient(pot)(s.coordinates, s.species, [s.natoms], e_ref, f_ref, s.cell[None])
    _, g_ref = ani_ref.loss_and_grads(s.coordinates, s.species, [s.natoms], W[0], CFG, MCFG, e_ref, f_ref,
                                      cells=s.cell[None])
    assert rel_err(g, g_ref) < REL_TOL


def test_gradient_entries_match_finite_differences(cuda_device):
    """Central differences of the FP64 loss, step 1e-4, on one entry of every
    kernel and bias of the hydrogen network."""
    xyz, sp, nat = batch(6, seed=45)
    W = init_weights(CFG, MCFG, seed=9, bias_std=0.05)
    e_ref, f_ref = teacher_targets(xyz, sp, nat)
    pot = ANIPotential(precision="fp32", device=cuda_device, weights=W)
    _, g = LossGradient(pot, dtype=torch.float64)(xyz, sp, nat, e_ref, f_ref)
    graph = ani_ref.Graph(xyz, nat, None, None, CFG.radial_cutoff, CFG.angular_cutoff)
    model = W[0]
    h = 1e-4
    for layer in range(4):
        for which in range(2):
            arr = model["H"][layer][which]
            idx = np.unravel_index(int(np.argmax(np.abs(g["H"][layer][which]))), arr.shape)
            orig = arr[idx]
            arr[idx] = orig + h
            lp = ani_ref.loss_value(xyz, sp, nat, model, CFG, MCFG, e_ref, f_ref, graph=graph)
            arr[idx] = orig - h
            lm = ani_ref.loss_value(xyz, sp, nat, model, CFG, MCFG, e_ref, f_ref, graph=graph)
            arr[idx] = orig
            fd = (lp - lm) / (2 * h)
            got = g["H"][layer][which][idx]
            assert abs(fd - got) <= 1e-3 * abs(fd) + 1e-9, (layer, which, fd, got)


def test_replayed_gradient_equals_direct(cuda_device):
    """From the third call on one batch the pass is one CUDA-graph replay;
    its results must equal the direct evaluation at new positions."""
    xyz, sp, nat = batch(16, seed=47)
    W = init_weights(CFG, MCFG, seed=10, bias_std=0.05)
    e_ref, f_ref = teacher_targets(xyz, sp, nat)
    pot = ANIPotential(precision="fp32", device=cuda_device, weights=W)
    lg = LossGradient(pot)
    rng = np.random.default_rng(3)
    for k in range(4):
        x = xyz + rng.normal(scale=0.02, size=xyz.shape)
        terms, g = lg(x, sp, nat, e_ref, f_ref)
        ref_pot = ANIPotential(precision="fp32", device=cuda_device, weights=W, use_graphs=False)
        t2, g2 = LossGradient(ref_pot, use_graphs=False)(x, sp, nat, e_ref, f_ref)
        assert abs(terms.loss - t2.loss) <= 1e-6 * t2.loss, k
        a, b = flatten(g, CFG.species_order), flatten(g2, CFG.species_order)
        assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(b), k
    assert lg._rec is not None  # the later calls replayed the captured pass
