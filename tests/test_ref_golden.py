"""The oracle's pair search against fixtures made by the reference's own host
graph builders (``tests/golden/make_ref_golden.py`` runs FeNNol's
``GraphGenerator``, ``GraphFilter`` and ``GraphAngularExtension`` numpy code):
radial pair sets, angular sub-graphs and triplets must be identical."""

from pathlib import Path

import numpy as np
import pytest

from oracle import graph_fp32

GOLDEN = Path(__file__).parent / "golden"
CASES = sorted(p.stem[len("ref_"):] for p in GOLDEN.glob("ref_*.npz"))


def load(name):
    return dict(np.load(GOLDEN / f"ref_{name}.npz"))


def _rows(*cols):
    keys = []
    for c in reversed(cols):
        c2 = np.asarray(c).reshape(len(c), -1)
        keys.extend(c2[:, k] for k in reversed(range(c2.shape[1])))
    o = np.lexsort(keys) if len(cols[0]) else np.zeros(0, int)
    return [np.asarray(c)[o] for c in cols]


def oracle_graph(d, cutoff):
    cells = d.get("cells")
    return graph_fp32.pair_list(d["coordinates"], d["natoms"], cells, None, cutoff,
                                bool(d["minimum_image"]))


def test_fixtures_present():
    assert {"water64_mi", "water4k_mi", "molecules6", "two_boxes_mi", "water8_general",
            "boundary_mi", "boundary_general", "boundary_nopbc", "water648_skin"} <= set(CASES)


@pytest.mark.parametrize("name", CASES)
def test_oracle_pairs_equal_reference(name):
    d = load(name)
    r = oracle_graph(d, 5.2)
    assert np.array_equal(r["p1"], d["p1"]) and np.array_equal(r["p2"], d["p2"])
    assert np.array_equal(r["shift"], d["shift"].astype(np.int64))
    if "skin_p1" in d:
        s = oracle_graph(d, 5.2 + float(d["skin"]))
        assert np.array_equal(s["p1"], d["skin_p1"]) and np.array_equal(s["p2"], d["skin_p2"])
        assert np.array_equal(s["shift"], d["skin_shift"].astype(np.int64))


@pytest.mark.parametrize("name", CASES)
def test_oracle_angular_graph_and_triplets_equal_reference(name):
    d = load(name)
    nat = int(d["natoms"].sum())
    r = oracle_graph(d, 5.2)
    src, dst, sh, d12 = graph_fp32.symmetrize(r)
    keep = d12 < np.float32(3.5 ** 2)
    a_src, a_dst, a_sh = _rows(src[keep], dst[keep], sh[keep])
    assert np.array_equal(a_src, d["a_src"]) and np.array_equal(a_dst, d["a_dst"])
    assert np.array_equal(a_sh, d["a_shift"].astype(np.int64))
    # triplets: unordered pairs of angular edges that share their source
    t_src, t_dst, t_c = graph_fp32.angular_triplets(src[keep], nat)
    assert np.array_equal(np.bincount(t_c, minlength=nat), d["t_count"])
    if "t_c" in d:
        dj, dk = dst[keep][t_src], dst[keep][t_dst]
        sj, sk = sh[keep][t_src], sh[keep][t_dst]
        kj = np.column_stack([dj, sj])
        kk = np.column_stack([dk, sk])
        first = np.array([tuple(a) <= tuple(b) for a, b in zip(kj.tolist(), kk.tolist())], bool)
        lo = np.where(first[:, None], kj, kk)
        hi = np.where(first[:, None], kk, kj)
        got = _rows(t_c, lo[:, 0], lo[:, 1:], hi[:, 0], hi[:, 1:])
        want = [d["t_c"], d["t_j"], d["t_sj"].astype(np.int64), d["t_k"], d["t_sk"].astype(np.int64)]
        for g, w in zip(got, want):
            assert np.array_equal(g, w)
