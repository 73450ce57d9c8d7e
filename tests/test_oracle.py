"""CPU tests of the oracle itself: golden fixtures, finite differences,
invariances and the pair-set arithmetic (no GPU)."""

from pathlib import Path

import numpy as np
import pytest
import torch

from fennol_b200.params import AEVConfig, MLPConfig, init_weights
from fennol_b200.systems import molecule_batch, water_box
from oracle import ani_ref, graph_fp32

GOLDEN = Path(__file__).parent / "golden"
CFG, MCFG = AEVConfig(), MLPConfig()


@pytest.fixture(scope="module")
def weights():
    return init_weights(CFG, MCFG, seed=0)


def _checksum(W):
    return float(sum(np.sum(w) + np.sum(b) for m in W for L in m.values() for w, b in L))


def test_golden_water64_reproduced(weights):
    d = np.load(GOLDEN / "water64.npz")
    assert abs(_checksum(weights) - float(d["weight_checksum"])) < 1e-9
    r = ani_ref.energy_and_forces(d["coordinates"], d["species"], [192], weights, CFG, MCFG,
                                  cells=d["cell"][None], return_aev=True)
    g = r["graph"]
    assert np.array_equal(g.pairs["p1"], d["p1"]) and np.array_equal(g.pairs["p2"], d["p2"])
    assert np.array_equal(g.pairs["shift"], d["shift"])
    assert np.array_equal(g.pairs["d12"], d["d12"])
    assert len(g.angle_src) == int(d["n_triplets"])
    np.testing.assert_allclose(r["energy"], d["energy"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(r["forces"], d["forces"], rtol=0, atol=1e-11)
    np.testing.assert_allclose(r["aev"][:8], d["aev_rows"], rtol=0, atol=1e-12)


def test_golden_molecules_reproduced(weights):
    d = np.load(GOLDEN / "molecules6.npz")
    r = ani_ref.energy_and_forces(d["coordinates"], d["species"], d["natoms"], weights, CFG, MCFG)
    np.testing.assert_allclose(r["energy"], d["energy"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(r["forces"], d["forces"], rtol=0, atol=1e-11)


def test_forces_match_finite_differences(weights):
    mols = molecule_batch(2, seed=11)
    xyz = np.concatenate([m.coordinates for m in mols])
    sp = np.concatenate([m.species for m in mols])
    nat = [m.natoms for m in mols]
    r = ani_ref.energy_and_forces(xyz, sp, nat, weights, CFG, MCFG)
    h = 1e-4
    rng = np.random.default_rng(0)
    for _ in range(6):
        i = int(rng.integers(len(sp)))
        k = int(rng.integers(3))
        e = []
        for sgn in (1, -1):
            x = xyz.copy()
            x[i, k] += sgn * h
            e.append(ani_ref.energy_and_forces(x, sp, nat, weights, CFG, MCFG, graph=r["graph"],
                                               need_forces=False)["energy"].sum())
        fd = -(e[0] - e[1]) / (2 * h)
        assert abs(fd - r["forces"][i, k]) < 1e-6 * max(1.0, abs(fd))


def test_rotation_translation_invariance(weights):
    m = molecule_batch(1, seed=5)[0]
    r0 = ani_ref.energy_and_forces(m.coordinates, m.species, [m.natoms], weights, CFG, MCFG)
    th = 0.7
    R = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]])
    x = m.coordinates @ R.T + np.array([1.5, -2.0, 0.25])
    r1 = ani_ref.energy_and_forces(x, m.species, [m.natoms], weights, CFG, MCFG)
    assert abs(r1["energy"][0] - r0["energy"][0]) < 1e-10
    np.testing.assert_allclose(r1["forces"], r0["forces"] @ R.T, atol=1e-9)


def test_pair_list_against_float64_distances():
    s = water_box(5, seed=2)
    p = graph_fp32.pair_list(s.coordinates, [s.natoms], s.cell[None], None, 5.2, True)
    L = s.cell[0, 0]
    x = s.coordinates
    i, j = np.triu_indices(s.natoms, 1)
    v = x[j] - x[i]
    v -= L * np.round(v / L)
    d = np.sqrt((v ** 2).sum(-1))
    have = set(zip(p["p1"].tolist(), p["p2"].tolist()))
    must = set(zip(i[d < 5.2 - 1e-4].tolist(), j[d < 5.2 - 1e-4].tolist()))
    may = set(zip(i[d < 5.2 + 1e-4].tolist(), j[d < 5.2 + 1e-4].tolist()))
    assert must <= have <= may


def test_general_pbc_matches_minimum_image_for_large_box():
    s = water_box(5, seed=4)
    a = graph_fp32.pair_list(s.coordinates, [s.natoms], s.cell[None], None, 5.2, True)
    b = graph_fp32.pair_list(s.coordinates, [s.natoms], s.cell[None], None, 5.2, False)
    assert np.array_equal(a["p1"], b["p1"]) and np.array_equal(a["p2"], b["p2"])
    # same image: raw-coordinate vectors agree
    xa = s.coordinates[a["p2"]] - s.coordinates[a["p1"]] + a["shift"] @ s.cell
    xb = s.coordinates[b["p2"]] - s.coordinates[b["p1"]] + b["shift"] @ s.cell
    np.testing.assert_allclose(xa, xb, atol=1e-9)


def test_skin_filter_equals_direct_list():
    s = water_box(4, seed=7)
    skin = graph_fp32.pair_list(s.coordinates, [s.natoms], s.cell[None], None, 6.2, True)
    direct = graph_fp32.pair_list(s.coordinates, [s.natoms], s.cell[None], None, 5.2, True)
    f = graph_fp32.filter_pairs(skin, 5.2)
    for k in ("p1", "p2", "shift", "d12"):
        assert np.array_equal(f[k], direct[k])


def test_triplet_count():
    s = water_box(4, seed=1)
    g = ani_ref.Graph(s.coordinates, [s.natoms], s.cell[None])
    src = g.src[g.filter_indices]
    cnt = np.bincount(src, minlength=g.nat)
    assert len(g.angle_src) == int((cnt * (cnt - 1) // 2).sum())


def test_canonical_from_ell_roundtrip():
    s = water_box(3, seed=9)
    p = graph_fp32.pair_list(s.coordinates, [s.natoms], s.cell[None], None, 5.2, True)
    src, dst, sh, _ = graph_fp32.symmetrize(p)
    n = s.natoms
    cnt = np.bincount(src, minlength=n)
    cap = int(cnt.max())
    nj = np.zeros((n, cap), np.int64)
    ns = np.zeros((n, cap, 3), np.int64)
    fill = np.zeros(n, np.int64)
    for a, b, v in zip(src, dst, sh):
        nj[a, fill[a]] = b
        ns[a, fill[a]] = v
        fill[a] += 1
    c, sym = graph_fp32.canonical_from_ell(nj, ns, cnt)
    assert sym
    assert np.array_equal(c["p1"], p["p1"]) and np.array_equal(c["p2"], p["p2"])
    assert np.array_equal(c["shift"], p["shift"])


def test_float32_oracle_close_to_float64(weights):
    s = water_box(3, seed=3)
    r64 = ani_ref.energy_and_forces(s.coordinates, s.species, [s.natoms], weights, CFG, MCFG,
                                    cells=s.cell[None])
    r32 = ani_ref.energy_and_forces(s.coordinates, s.species, [s.natoms], weights, CFG, MCFG,
                                    cells=s.cell[None], dtype=torch.float32, graph=r64["graph"])
    assert abs(r32["energy"][0] - r64["energy"][0]) * 627.5 / s.natoms < 1e-4
    assert np.sqrt(((r32["forces"] - r64["forces"]) ** 2).mean()) * 627.5 < 0.05


def test_loss_parameter_gradients_match_finite_differences():
    """Second-order autograd of the energy + force loss (the training
    gradient) against central differences, FP64, step 1e-4."""
    from fennol_b200.params import AEVConfig, MLPConfig, init_weights
    from fennol_b200.systems import molecule_batch
    from oracle import ani_ref

    cfg, mcfg = AEVConfig(), MLPConfig()
    mols = molecule_batch(3, seed=31, nmin=8, nmax=14)
    xyz = np.concatenate([m.coordinates for m in mols])
    sp = np.concatenate([m.species for m in mols])
    nat = [m.natoms for m in mols]
    model = init_weights(cfg, mcfg, seed=3, bias_std=0.1)[0]
    teacher = init_weights(cfg, mcfg, seed=4)
    ref = ani_ref.energy_and_forces(xyz, sp, nat, teacher, cfg, mcfg)
    graph = ani_ref.Graph(xyz, nat, None, None, cfg.radial_cutoff, cfg.angular_cutoff)
    loss, grads = ani_ref.loss_and_grads(xyz, sp, nat, model, cfg, mcfg, ref["energy"], ref["forces"],
                                         graph=graph)
    assert abs(loss - ani_ref.loss_value(xyz, sp, nat, model, cfg, mcfg, ref["energy"], ref["forces"],
                                         graph=graph)) < 1e-12 * max(1.0, loss)
    rng = np.random.default_rng(0)
    present = sorted({cfg.species_order[k] for k in cfg.species_index(sp)})
    h = 1e-4
    for _ in range(10):
        sym = present[int(rng.integers(len(present)))]
        layer = int(rng.integers(4))
        which = int(rng.integers(2))
        arr = model[sym][layer][which]
        idx = tuple(int(rng.integers(n)) for n in arr.shape)
        orig = arr[idx]
        arr[idx] = orig + h
        lp = ani_ref.loss_value(xyz, sp, nat, model, cfg, mcfg, ref["energy"], ref["forces"], graph=graph)
        arr[idx] = orig - h
        lm = ani_ref.loss_value(xyz, sp, nat, model, cfg, mcfg, ref["energy"], ref["forces"], graph=graph)
        arr[idx] = orig
        fd = (lp - lm) / (2 * h)
        g = grads[sym][layer][which][idx]
        assert abs(fd - g) <= 1e-5 * abs(g) + 1e-9 * max(1.0, loss), (sym, layer, which, idx, fd, g)


def test_virial_of_a_molecule_is_minus_sum_x_outer_f():
    """Without a cell the strain derivative equals sum_i x_i (x) dE/dx_i."""
    from fennol_b200.params import AEVConfig, MLPConfig, init_weights
    from fennol_b200.systems import molecule_batch
    from oracle import ani_ref

    cfg, mcfg = AEVConfig(), MLPConfig()
    mols = molecule_batch(2, seed=17, nmin=10, nmax=16)
    xyz = np.concatenate([m.coordinates for m in mols])
    sp = np.concatenate([m.species for m in mols])
    nat = [m.natoms for m in mols]
    W = init_weights(cfg, mcfg, seed=2)
    r = ani_ref.energy_forces_virial(xyz, sp, nat, W, cfg, mcfg)
    off = np.concatenate([[0], np.cumsum(nat)])
    for b in range(len(nat)):
        x, f = xyz[off[b]:off[b + 1]], r["forces"][off[b]:off[b + 1]]
        np.testing.assert_allclose(r["virial"][b], -np.einsum("ia,ib->ab", x, f), rtol=1e-10, atol=1e-12)
