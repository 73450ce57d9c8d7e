"""The FeNNol-compatible API driving the CUDA path: energies and forces
against the FP64 oracle and against the direct host API, the edge-list view
of the graphs against the oracle's pair lists, the fixed-capacity
(``process`` + ``check_reallocate``) path and the skin update."""

from collections import OrderedDict
from pathlib import Path

import numpy as np
import pytest
import torch

from fennol_b200.fennix import FENNIX, graph_edges
from fennol_b200.params import AEVConfig, MLPConfig, variables_to_weights
from fennol_b200.potential import ANIPotential, HARTREE_TO_KCALMOL
from fennol_b200.systems import molecule_batch, water_box
from oracle import ani_ref, graph_fp32
from test_fennix_api import ani_modules, ani_preprocessing

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).parent / "golden"
FORCE_RMSE_TOL = 0.05   # kcal/mol/A against FP64
ENERGY_TOL = 1e-4       # kcal/mol/atom against FP64


def make_model(precision="fp32", **kw):
    return FENNIX(5.2, ani_modules(), ani_preprocessing(), energy_terms=["energy"],
                  precision=precision, **kw)


def weights_of(m):
    return variables_to_weights([m.variables], m.aev_config.species_order, "energy")


def test_water64_golden_through_fennix(cuda_device):
    d = np.load(GOLDEN / "water64.npz")
    m = make_model(rng_key=0)
    e, f, out = m.energy_and_forces(species=d["species"], coordinates=d["coordinates"],
                                    natoms=np.array([192]), cells=d["cell"][None],
                                    flags={"minimum_image": True})
    de = abs(float(e[0]) - float(d["energy"][0])) * HARTREE_TO_KCALMOL / 192
    rmse = np.sqrt(np.mean((f.cpu().numpy() - d["forces"]) ** 2)) * HARTREE_TO_KCALMOL
    assert de <= ENERGY_TOL and rmse <= FORCE_RMSE_TOL, (de, rmse)
    assert out["energy"].shape == (192,)
    assert abs(float(out["energy"].sum()) - float(e[0])) < 1e-9


@pytest.mark.parametrize("precision", ["fp32", "bf16x2"])
def test_same_as_host_api(cuda_device, precision):
    mols = molecule_batch(6, seed=4)
    sp = np.concatenate([s.species for s in mols])
    xyz = np.concatenate([s.coordinates for s in mols])
    nat = np.array([s.natoms for s in mols])
    m = make_model(precision)
    e, f, _ = m.energy_and_forces(species=sp, coordinates=xyz, natoms=nat)
    pot = ANIPotential(precision=precision, device=cuda_device, weights=weights_of(m))
    e2, f2 = pot.energy_and_forces(xyz, sp, nat)
    np.testing.assert_allclose(e.cpu().numpy(), e2.cpu().numpy(), rtol=0, atol=1e-9)
    np.testing.assert_allclose(f.cpu().numpy(), f2.cpu().numpy(), rtol=0, atol=1e-7)


@pytest.mark.parametrize("mi", [True, False])
def test_graph_edges_match_oracle_pairs(cuda_device, mi):
    s = water_box(8, seed=5)
    m = make_model()
    flags = {"minimum_image": True} if mi else {}
    inputs = m.preprocess(species=s.species, coordinates=s.coordinates, natoms=np.array([s.natoms]),
                          cells=s.cell[None], flags=flags)
    for key, rc in (("graph", 5.2), ("graph_angle", 3.5)):
        ed = graph_edges(inputs, key)
        ref = graph_fp32.pair_list(s.coordinates, [s.natoms], s.cell[None], None, rc, mi)
        src, dst, sh, _ = graph_fp32.symmetrize(ref)
        got = {tuple(r) for r in np.column_stack([ed["edge_src"], ed["edge_dst"],
                                                  ed["pbc_shifts"].astype(np.int64)]).tolist()}
        want = {tuple(r) for r in np.column_stack([src, dst, sh]).tolist()}
        assert got == want and len(got) == ed["edge_src"].shape[0], key
        assert np.all(ed["d12"] < rc ** 2 * (1 + 1e-5))


def test_gpu_preprocessing_reallocates(cuda_device):
    s = water_box(8, seed=6)
    m = make_model()
    args = dict(species=s.species, coordinates=s.coordinates, natoms=np.array([s.natoms]),
                cells=s.cell[None], flags={"minimum_image": True})
    e0, f0, _ = m.energy_and_forces(**args)
    layers = list(m.preproc_state["layers_state"])
    layers[0] = {**layers[0], "max_neigh": 16}
    layers[1] = {**layers[1], "max_neigh": 8}
    m.preproc_state = {**m.preproc_state, "layers_state": tuple(layers)}
    e1, f1, _ = m.energy_and_forces(gpu_preprocessing=True, **args)
    assert m.preproc_state["layers_state"][0]["max_neigh"] > 16
    assert m.preproc_state["layers_state"][1]["max_neigh"] > 8
    np.testing.assert_allclose(e1.cpu().numpy(), e0.cpu().numpy(), rtol=0, atol=1e-9)
    np.testing.assert_allclose(f1.cpu().numpy(), f0.cpu().numpy(), rtol=0, atol=1e-7)


def test_sized_call_regrows_on_denser_input(cuda_device):
    """A sized model launches its graph layers at the stored capacities and
    checks their overflow words with the evaluation's status; a denser input
    overflows them, and the call reruns through the growing path."""
    s = water_box(8, seed=11)
    m = make_model()
    args = dict(species=s.species, natoms=np.array([s.natoms]), flags={"minimum_image": True})
    e0, f0, _ = m.energy_and_forces(coordinates=s.coordinates, cells=s.cell[None], **args)
    e0b, f0b, _ = m.energy_and_forces(coordinates=s.coordinates, cells=s.cell[None], **args)
    # the force adjoint accumulates with float32 atomics: the order of the
    # additions, and so the last bits, can differ between two evaluations
    assert float(e0b[0]) == float(e0[0])
    np.testing.assert_allclose(f0b.cpu().numpy(), f0.cpu().numpy(), rtol=0, atol=1e-6)
    caps = [dict(x) for x in m.preproc_state["layers_state"]]
    squeeze = 0.82
    dense = dict(coordinates=(s.coordinates * squeeze).astype(np.float32),
                 cells=(s.cell * squeeze)[None], **args)
    e1, f1, _ = m.energy_and_forces(**dense)
    grown = m.preproc_state["layers_state"]
    assert grown[0]["max_neigh"] > caps[0]["max_neigh"]
    assert grown[1]["max_neigh"] >= caps[1]["max_neigh"]
    fresh = make_model()
    e2, f2, _ = fresh.energy_and_forces(**dense)
    np.testing.assert_allclose(e1.cpu().numpy(), e2.cpu().numpy(), rtol=0, atol=1e-9)
    np.testing.assert_allclose(f1.cpu().numpy(), f2.cpu().numpy(), rtol=0, atol=1e-6)


@pytest.mark.parametrize("kind", ["box", "molecules"])
def test_graph_replay_equals_eager_calls(cuda_device, kind):
    """Sized calls replay one captured CUDA graph per layout; each call's
    outputs equal those of the kernel-by-kernel path on the same inputs, and
    the returned tensors are the caller's own (not rewritten by the next
    replay)."""
    if kind == "box":
        s = water_box(8, seed=12)
        sp, xyz0, nat = s.species, s.coordinates, np.array([s.natoms])
        extra = dict(cells=s.cell[None], flags={"minimum_image": True})
    else:
        mols = molecule_batch(5, seed=12)
        sp = np.concatenate([m.species for m in mols])
        xyz0 = np.concatenate([m.coordinates for m in mols])
        nat = np.array([m.natoms for m in mols])
        extra = {}
    graph, eager = make_model("f16x3x1"), make_model("f16x3x1")
    eager.use_cuda_graphs = False
    rng = np.random.default_rng(3)
    kept = []
    for call in range(4):
        xyz = (xyz0 + rng.normal(0.0, 0.02, xyz0.shape)).astype(np.float32)
        args = dict(species=sp, coordinates=xyz, natoms=nat, **extra)
        e1, f1, o1 = graph.energy_and_forces(**args)
        e2, f2, o2 = eager.energy_and_forces(**args)
        np.testing.assert_array_equal(e1.cpu().numpy(), e2.cpu().numpy())
        np.testing.assert_allclose(f1.cpu().numpy(), f2.cpu().numpy(), rtol=0, atol=1e-6)
        np.testing.assert_array_equal(o1["energy"].cpu().numpy(), o2["energy"].cpu().numpy())
        assert o1["coordinates"] is xyz
        kept.append((e1, f1.clone(), f1))
    assert len(graph._graphs) == 1
    for e, f_copy, f in kept:
        assert torch.equal(f, f_copy)
    # the other entry points replay graphs of their own
    args = dict(species=sp, coordinates=xyz0.astype(np.float32), natoms=nat, **extra)
    for _ in range(3):
        t1, _ = graph.total_energy(**args)
        emb1 = graph(**args)["embedding"]
        v1 = graph.energy_and_forces_and_virial(**args)
    t2, _ = eager.total_energy(**args)
    emb2 = eager(**args)["embedding"]
    v2 = eager.energy_and_forces_and_virial(**args)
    np.testing.assert_array_equal(t1.cpu().numpy(), t2.cpu().numpy())
    np.testing.assert_array_equal(emb1.cpu().numpy(), emb2.cpu().numpy())
    np.testing.assert_array_equal(v1[0].cpu().numpy(), v2[0].cpu().numpy())
    np.testing.assert_allclose(v1[2].cpu().numpy(), v2[2].cpu().numpy(), rtol=1e-5, atol=1e-6)
    assert len(graph._graphs) == 4


def test_skin_update_matches_fresh_build(cuda_device):
    s = water_box(8, seed=7)
    m = make_model()
    layers = list(m.preprocessing.init()["layers_state"])
    layers[0] = {**layers[0], "nblist_skin": 1.0}
    m.preproc_state = {**m.preproc_state, "layers_state": tuple(layers)}
    args = dict(species=s.species, natoms=np.array([s.natoms]), cells=s.cell[None],
                flags={"minimum_image": True})
    inputs = m.preprocess(coordinates=s.coordinates, **args)
    rng = np.random.default_rng(0)
    # at most 0.25*sqrt(3) = 0.43 A per atom: pairs approach by less than the 1 A skin
    moved = (s.coordinates + rng.uniform(-0.25, 0.25, s.coordinates.shape)).astype(np.float32)
    inputs = {**inputs, "coordinates": moved,
              "_coords": torch.tensor(moved, device=cuda_device)}
    inputs = m.preprocessing.update_skin(inputs)
    ed = graph_edges(inputs, "graph")
    ref = graph_fp32.pair_list(moved, [s.natoms], s.cell[None], None, 5.2, True)
    src, dst, sh, _ = graph_fp32.symmetrize(ref)
    got = {tuple(r) for r in np.column_stack([ed["edge_src"], ed["edge_dst"],
                                              ed["pbc_shifts"].astype(np.int64)]).tolist()}
    want = {tuple(r) for r in np.column_stack([src, dst, sh]).tolist()}
    assert got == want


def test_units_total_energy_and_embedding(cuda_device):
    d = np.load(GOLDEN / "water64.npz")
    m = make_model(rng_key=0)
    args = dict(species=d["species"], coordinates=d["coordinates"], natoms=np.array([192]),
                cells=d["cell"][None], flags={"minimum_image": True})
    e_ha, f_ha, _ = m.energy_and_forces(**args)
    e_kc, f_kc, _ = m.energy_and_forces(unit="kcalpermol", **args)
    np.testing.assert_allclose(e_kc.cpu().numpy(), e_ha.cpu().numpy() * HARTREE_TO_KCALMOL, rtol=1e-12)
    # two evaluations: the atomic force sums may round differently (float32)
    np.testing.assert_allclose(f_kc.cpu().numpy(), f_ha.cpu().numpy() * HARTREE_TO_KCALMOL,
                               rtol=1e-5, atol=1e-4)
    e_only, _ = m.total_energy(**args)
    assert abs(float(e_only[0]) - float(e_ha[0])) < 1e-9
    out = m(**args)
    emb = out["embedding"].cpu().numpy()[:8]
    np.testing.assert_allclose(emb, d["aev_rows"], rtol=1e-4, atol=2e-5)


def test_loaded_model_same_results(cuda_device, tmp_path):
    mols = molecule_batch(4, seed=9)
    sp = np.concatenate([s.species for s in mols])
    xyz = np.concatenate([s.coordinates for s in mols])
    nat = np.array([s.natoms for s in mols])
    m = make_model(rng_key=5)
    m.save(tmp_path / "m.fnx")
    m2 = FENNIX.load(tmp_path / "m.fnx", precision="fp32")
    e, f, _ = m.energy_and_forces(species=sp, coordinates=xyz, natoms=nat)
    e2, f2, _ = m2.energy_and_forces(species=sp, coordinates=xyz, natoms=nat)
    assert torch.equal(e, e2)
    np.testing.assert_allclose(f.cpu().numpy(), f2.cpu().numpy(), rtol=0, atol=1e-6)
    r = ani_ref.energy_and_forces(xyz, sp, nat, weights_of(m), AEVConfig(), MLPConfig())
    de = np.abs(e.cpu().numpy() - r["energy"]).max() * HARTREE_TO_KCALMOL / nat.min()
    assert de <= ENERGY_TOL
