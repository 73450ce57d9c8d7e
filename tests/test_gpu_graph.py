"""GPU parity of the neighbour search: the pair set must be bit-identical to
the reference's float32 numpy builder (restated in oracle.graph_fp32)."""

from pathlib import Path

import numpy as np
import pytest
import torch

from fennol_b200 import _lib
from fennol_b200.params import AEVConfig
from fennol_b200.potential import ANIPotential, GraphBuffers, unpack_shifts
from fennol_b200.systems import molecule_batch, water_box
from oracle import graph_fp32

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).parent / "golden"


@pytest.fixture(scope="module")
def pot(cuda_device):
    return ANIPotential(precision="fp32", device=cuda_device)


def _gpu_pairs(pot, xyz, sp, nat, cells, cutoff, minimum_image=True):
    prev, pot.minimum_image = pot.minimum_image, minimum_image
    try:
        nj, ns, nn, _ = pot.neighbor_lists(xyz, sp, nat, cells, cutoff)
    finally:
        pot.minimum_image = prev
    canon, sym = graph_fp32.canonical_from_ell(nj, unpack_shifts(ns), nn)
    return canon, sym, nj, ns, nn


def _same(canon, ref):
    return (np.array_equal(canon["p1"], ref["p1"]) and np.array_equal(canon["p2"], ref["p2"])
            and np.array_equal(canon["shift"], ref["shift"]))


def test_golden_water64_pairs(pot):
    d = np.load(GOLDEN / "water64.npz")
    canon, sym, *_ = _gpu_pairs(pot, d["coordinates"], d["species"], [192], d["cell"][None], 5.2)
    assert sym
    ref = {"p1": d["p1"], "p2": d["p2"], "shift": d["shift"].astype(np.int64)}
    assert _same(canon, ref)
    canon, sym, *_ = _gpu_pairs(pot, d["coordinates"], d["species"], [192], d["cell"][None], 5.2,
                                minimum_image=False)
    ref = {"p1": d["gen_p1"], "p2": d["gen_p2"], "shift": d["gen_shift"].astype(np.int64)}
    assert sym and _same(canon, ref)


@pytest.mark.parametrize("n_side,seed,mi", [(8, 0, True), (8, 1, False), (11, 2, True), (16, 3, True)])
def test_water_box_pairs_cell_list(pot, n_side, seed, mi):
    s = water_box(n_side, seed=seed)
    for rc in (5.2, 6.2, 3.5):
        ref = graph_fp32.pair_list(s.coordinates, [s.natoms], s.cell[None], None, rc, mi)
        canon, sym, *_ = _gpu_pairs(pot, s.coordinates, s.species, [s.natoms], s.cell[None], rc, mi)
        assert sym, (n_side, rc)
        assert _same(canon, ref), (n_side, rc, len(canon["p1"]), len(ref["p1"]))


def test_crowded_stencil_fallback_pairs(pot):
    """A box whose stencils partly hold more candidates than a block stages
    (a dense 4 A clump of 700 extra atoms): those cells take the per-atom
    gather path, the others the staged one; the pair set stays the oracle's."""
    s = water_box(8, seed=4)
    rng = np.random.default_rng(4)
    corner = s.coordinates.min(0) + 3.0
    clump = (corner + rng.uniform(0.0, 4.0, (700, 3))).astype(np.float32)
    xyz = np.concatenate([s.coordinates, clump]).astype(np.float32)
    sp = np.concatenate([s.species, np.full(700, 1, s.species.dtype)])
    for mi in (True, False):
        ref = graph_fp32.pair_list(xyz, [len(sp)], s.cell[None], None, 5.2, mi)
        canon, sym, *_ = _gpu_pairs(pot, xyz, sp, [len(sp)], s.cell[None], 5.2, mi)
        assert sym and _same(canon, ref), (mi, len(canon["p1"]), len(ref["p1"]))


def test_molecule_batch_pairs(pot):
    mols = molecule_batch(20, seed=4)
    xyz = np.concatenate([m.coordinates for m in mols])
    sp = np.concatenate([m.species for m in mols])
    nat = [m.natoms for m in mols]
    ref = graph_fp32.pair_list(xyz, nat, None, None, 5.2)
    canon, sym, *_ = _gpu_pairs(pot, xyz, sp, nat, None, 5.2)
    assert sym and _same(canon, ref)


def test_mixed_batch_pairs(pot):
    """A periodic box and molecules in one launch: pairs never cross systems."""
    box = water_box(8, seed=5)
    mols = molecule_batch(3, seed=6)
    systems = [mols[0], box, mols[1], mols[2]]
    xyz = np.concatenate([s.coordinates for s in systems])
    sp = np.concatenate([s.species for s in systems])
    nat = [s.natoms for s in systems]
    cells = [None, box.cell, None, None]
    canon, sym, *_ = _gpu_pairs(pot, xyz, sp, nat, cells, 5.2)
    assert sym
    off = np.concatenate([[0], np.cumsum(nat)])
    parts = []
    for b, s in enumerate(systems):
        r = graph_fp32.pair_list(s.coordinates, [s.natoms], None if cells[b] is None else cells[b][None],
                                 None, 5.2)
        parts.append((r["p1"] + off[b], r["p2"] + off[b], r["shift"]))
    ref = {"p1": np.concatenate([p[0] for p in parts]), "p2": np.concatenate([p[1] for p in parts]),
           "shift": np.concatenate([p[2] for p in parts])}
    o = np.lexsort((ref["shift"][:, 2], ref["shift"][:, 1], ref["shift"][:, 0], ref["p2"], ref["p1"]))
    ref = {k: v[o] for k, v in ref.items()}
    assert _same(canon, ref)


def test_boundary_pairs_exactly_at_cutoff_and_cell_faces(pot):
    """Atoms at x = 0 and x = 5.2f: d^2 = fl(5.2f^2) = 27.039997 < fl(27.04); pairs
    at 5.2000003; atoms on bin faces and at the box edge (wrap)."""
    L = 31.2  # 6 bins of 5.2 A: many atoms sit exactly on bin faces
    f = np.float32
    pts = []
    for k in range(6):
        base = f(k * 5.2)
        pts.append([base, 1.0, 1.0])
        pts.append([f(base + f(5.2)), 1.0, 1.0])
        pts.append([f(base + np.nextafter(f(5.2), f(10))), 3.0, 1.0])
        pts.append([base, 3.0, 1.0])
    pts.append([f(L), 7.0, 7.0])
    pts.append([f(0.0), 7.0, 7.0])
    pts.append([f(-1e-7), 12.0, 12.0])
    pts.append([f(L - 5.2), 12.0, 12.0])
    xyz = np.array(pts, dtype=np.float64)
    sp = np.full(len(pts), 6)
    cell = np.eye(3) * L
    for mi in (True, False):
        ref = graph_fp32.pair_list(xyz, [len(pts)], cell[None], None, 5.2, mi)
        canon, sym, *_ = _gpu_pairs(pot, xyz, sp, [len(pts)], cell[None], 5.2, mi)
        assert sym and _same(canon, ref), mi
    ref = graph_fp32.pair_list(xyz, [len(pts)], None, None, 5.2)
    canon, sym, *_ = _gpu_pairs(pot, xyz, sp, [len(pts)], None, 5.2)
    assert sym and _same(canon, ref)


def test_small_box_all_pairs_path(pot):
    """12.42 A box with a 6.2 A skin cutoff: fewer than 3 bins -> all-pairs path."""
    s = water_box(4, seed=8)
    for mi in (True, False):
        ref = graph_fp32.pair_list(s.coordinates, [s.natoms], s.cell[None], None, 6.2, mi)
        canon, sym, *_ = _gpu_pairs(pot, s.coordinates, s.species, [s.natoms], s.cell[None], 6.2, mi)
        assert sym and _same(canon, ref)


def test_overflow_reports_and_regrows(pot, cuda_device):
    s = water_box(6, seed=9)
    lay = pot.layout(s.species, [s.natoms], s.cell[None])
    coords = torch.tensor(s.coordinates, dtype=torch.float32, device=cuda_device)
    status = torch.zeros(8, dtype=torch.int32, device=cuda_device)
    g = GraphBuffers(lay, 5.2, 0.0, 16, 16)
    g.build(lay, coords, status, torch.cuda.current_stream().cuda_stream)
    st = status.cpu().numpy()
    assert st[_lib.ST_NBR_OVERFLOW] == 1 and st[_lib.ST_NBR_MAXCOUNT] > 16
    assert int(g.nbr_n.max()) == 16  # rows clamped to the capacity, nothing written past it
    ref = graph_fp32.pair_list(s.coordinates, [s.natoms], s.cell[None], None, 5.2)
    canon, sym, *_ = _gpu_pairs(pot, s.coordinates, s.species, [s.natoms], s.cell[None], 5.2)
    assert sym and _same(canon, ref)


def test_skin_filter_matches_direct_list(pot, cuda_device):
    s = water_box(10, seed=10)
    lay = pot.layout(s.species, [s.natoms], s.cell[None])
    coords = torch.tensor(s.coordinates, dtype=torch.float32, device=cuda_device)
    status = torch.zeros(8, dtype=torch.int32, device=cuda_device)
    g = GraphBuffers(lay, 5.2, 1.0, 160, 128)
    st_ = torch.cuda.current_stream().cuda_stream
    g.build(lay, coords, status, st_)
    # move atoms a little (below half the skin), then filter the skin list
    rng = np.random.default_rng(0)
    moved = s.coordinates + rng.uniform(-0.2, 0.2, s.coordinates.shape)
    coords2 = torch.tensor(moved, dtype=torch.float32, device=cuda_device)
    g.filter(lay, coords2, status, st_)
    assert int(status[_lib.ST_NBR_OVERFLOW]) == 0 and int(status[_lib.ST_FILTER_OVERFLOW]) == 0
    canon, sym = graph_fp32.canonical_from_ell(g.rad_j.cpu().numpy(), unpack_shifts(g.rad_s.cpu().numpy()),
                                               g.rad_n.cpu().numpy())
    # reference update_skin semantics: the skin shifts are kept, d^2 recomputed
    skin = graph_fp32.pair_list(s.coordinates, [s.natoms], s.cell[None], None, 6.2)
    x32 = moved.astype(np.float32)
    vec = (x32[skin["p2"]] - x32[skin["p1"]]) + np.dot(skin["shift"].astype(np.float32),
                                                        s.cell.astype(np.float32))
    d12 = (vec ** 2).sum(-1)
    keep = d12 < 5.2 ** 2
    ref = {"p1": skin["p1"][keep], "p2": skin["p2"][keep], "shift": skin["shift"][keep]}
    assert sym and _same(canon, ref)


# ---- fixtures made by the reference's own host graph builders ------------------------

REF_CASES = sorted(p.stem[len("ref_"):] for p in GOLDEN.glob("ref_*.npz"))


def _directed(nj, ns, nn):
    """Directed edges (i, j, shift) of ELL rows, sorted."""
    rows = np.repeat(np.arange(nn.shape[0]), nn)
    cols = np.concatenate([np.arange(k) for k in nn]) if nn.size else np.zeros(0, int)
    j = nj[rows, cols].astype(np.int64)
    s = unpack_shifts(ns[rows, cols]).astype(np.int64)
    o = np.lexsort((s[:, 2], s[:, 1], s[:, 0], j, rows))
    return rows[o], j[o], s[o]


@pytest.mark.parametrize("name", REF_CASES)
def test_rows_equal_reference_builder(pot, name):
    """Radial pair set, the skin list (if any), the directed angular
    sub-graph and the number of triplets per centre, against FeNNol's own
    GraphGenerator / GraphFilter / GraphAngularExtension (bit-exact)."""
    d = dict(np.load(GOLDEN / f"ref_{name}.npz"))
    cells = d.get("cells")
    nat = [int(v) for v in d["natoms"]]
    mi = bool(d["minimum_image"])
    canon, sym, *_ = _gpu_pairs(pot, d["coordinates"], d["species"], nat, cells, 5.2, mi)
    ref = {"p1": d["p1"], "p2": d["p2"], "shift": d["shift"].astype(np.int64)}
    assert sym and _same(canon, ref), name
    if "skin_p1" in d:
        canon, sym, *_ = _gpu_pairs(pot, d["coordinates"], d["species"], nat, cells, 5.2 + float(d["skin"]), mi)
        ref = {"p1": d["skin_p1"], "p2": d["skin_p2"], "shift": d["skin_shift"].astype(np.int64)}
        assert sym and _same(canon, ref), name
    *_, nj, ns, nn = _gpu_pairs(pot, d["coordinates"], d["species"], nat, cells, 3.5, mi)
    src, dst, sh = _directed(nj, ns, nn)
    assert np.array_equal(src, d["a_src"]) and np.array_equal(dst, d["a_dst"])
    assert np.array_equal(sh, d["a_shift"].astype(np.int64))
    # the AEV kernels form every unordered pair of a centre's angular neighbours
    assert np.array_equal(nn.astype(np.int64) * (nn - 1) // 2, d["t_count"])


@pytest.mark.parametrize("name", ["water64_mi", "molecules6", "water8_general", "two_boxes_mi"])
def test_aev_on_reference_graphs(cuda_device, name):
    """AEV rows of the CUDA kernels on the fixture geometries against the
    FP64 oracle, whose pairs and triplets equal the reference builder's
    (tests/test_ref_golden.py): a missing or extra triplet would move a row
    far beyond the float32 tolerance."""
    from fennol_b200.params import MLPConfig
    from oracle import ani_ref

    d = dict(np.load(GOLDEN / f"ref_{name}.npz"))
    cells = d.get("cells")
    nat = [int(v) for v in d["natoms"]]
    mi = bool(d["minimum_image"])
    p = ANIPotential(precision="fp32", device=cuda_device, minimum_image=mi)
    p.energy_and_forces(d["coordinates"], d["species"], nat, cells)
    layout, g, ws = next(iter(p._cache.values()))
    got = ws.x.float().cpu().numpy()[layout.atom_row_host, :1008]
    r = ani_ref.energy_and_forces(d["coordinates"], d["species"], nat, p.weights, AEVConfig(), MLPConfig(),
                                  cells=cells, minimum_image=mi, need_forces=False, return_aev=True)
    np.testing.assert_allclose(got, r["aev"], rtol=1e-4, atol=2e-5)
