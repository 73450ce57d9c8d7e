"""CPU tests of the C-ABI library: it loads, exports every declared symbol,
and its host-only entry points and argument checks behave (no GPU work)."""

import ctypes as C

import numpy as np
import pytest

from fennol_b200 import _lib
from fennol_b200.params import AEVConfig
from fennol_b200.potential import aev_params, BatchLayout


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = _lib.declared_symbols()
    assert len(declared) >= 15
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(_lib._SIGNATURES)
    assert b"sm_100a" in lib.fennol_version()


def _plan(mode, recip, cutoff):
    n = len(mode)
    grid = np.zeros((n, 4), np.int32)
    nrep = np.zeros((n, 3), np.int32)
    mode = np.asarray(mode, np.int32)
    recip = np.asarray(recip, np.float32).reshape(n, 9)
    total = _lib.load().fennol_graph_plan(n, mode.ctypes.data, recip.ctypes.data, cutoff,
                                          grid.ctypes.data, nrep.ctypes.data)
    return total, grid, nrep


def test_graph_plan_cells_and_allpairs():
    L = [49.7, 12.42, 30.0]
    recip = [np.eye(3) / l for l in L]
    total, grid, nrep = _plan([1, 1, 0], recip, 6.2)
    assert tuple(grid[0, :3]) == (8, 8, 8)        # 49.7 / 6.2 = 8.02 bins
    assert tuple(grid[1, :3]) == (0, 0, 0)        # 12.42 A box: all pairs
    assert tuple(grid[2, :3]) == (0, 0, 0)        # no cell: all pairs
    assert total == 512
    assert grid[0, 3] == 0
    assert tuple(nrep[1]) == (1, 1, 1)
    # bins are wider than the cutoff
    assert 49.7 / 8 > 6.2


def test_graph_plan_rejects_bad_arguments():
    lib = _lib.load()
    assert lib.fennol_graph_plan(1, None, None, 5.2, None, None) == _lib.ERR_INVALID


def test_entry_points_validate_before_launching():
    lib = _lib.load()
    # null device pointers are rejected on the host; nothing is launched
    assert lib.fennol_graph_build(None, 10, None, 1, None, None, None, None, None, None, 0, 5.2, 64,
                                  None, None, None, None, None, 0, None, None) == _lib.ERR_INVALID
    assert lib.fennol_graph_filter(None, 10, None, None, None, None, None, 8, 5.2, 8, None, None,
                                   None, None, None) == _lib.ERR_INVALID
    p = aev_params(AEVConfig())
    assert lib.fennol_aev_forward(None, 10, None, None, None, None, None, 8, C.byref(p), None, 0,
                                  None, None, 1024, None, None) == _lib.ERR_INVALID
    assert lib.fennol_mlp_energy_grad(7, 128, 1, None, None, None, None, None, None, None, None, 0,
                                      None) == _lib.ERR_INVALID
    assert lib.fennol_md_step(10, -1.0, None, None, None, None, 1.0, 1.0, None, 0, 0, None, None,
                              None, None, 0.5, None, None) == _lib.ERR_INVALID
    # empty inputs are a no-op success
    assert lib.fennol_pack_atoms(None, None, 0, None, None) == _lib.OK


def test_aev_length_and_unsupported_parameters():
    lib = _lib.load()
    p = aev_params(AEVConfig())
    assert lib.fennol_aev_length(C.byref(p)) == 1008
    p.angle_sections = 3
    assert lib.fennol_aev_length(C.byref(p)) == -1
    p = aev_params(AEVConfig(species_order=("H", "C", "N", "O")))
    assert lib.fennol_aev_length(C.byref(p)) == 4 * 16 + 10 * 32


def test_workspace_queries_grow():
    lib = _lib.load()
    a = lib.fennol_graph_workspace_bytes(1000, 64)
    b = lib.fennol_graph_workspace_bytes(100000, 4096)
    assert 0 < a < b


def test_batch_layout_species_tiles():
    sp = np.array([0, 3, 3, 0, 0, 1] * 50, dtype=np.int32)
    cell = np.eye(3) * 20.0
    lay = BatchLayout(sp, [100, 200], [cell, None], True, device="cpu")
    rows = lay.atom_row_host
    assert len(set(rows.tolist())) == sp.size
    assert lay.rows % 128 == 0 and lay.ntiles == int(lay.t_tile_row.numel())
    # every row of a tile holds one species; rows follow input order inside a species
    for s in range(4):
        idx = np.nonzero(sp == s)[0]
        if idx.size:
            assert np.all(np.diff(rows[idx]) == 1)
    tiles = list(zip(lay.t_tile_species.tolist(), lay.t_tile_row.tolist()))
    for i in range(sp.size):
        t = [k for k, (s, r) in enumerate(tiles) if r <= rows[i] < r + 128]
        assert len(t) == 1 and tiles[t[0]][0] == sp[i]
    assert lay.mode_host.tolist() == [_lib.PBC_MINIMUM_IMAGE, _lib.PBC_NONE]
    assert lay.plan(5.2)[2] == 27   # 20 A / 5.2 A -> 3 bins per axis
    assert lay.plan(7.0)[2] == 0    # 20 A / 7 A -> 2 bins: all-pairs path


def test_serving_host_helpers():
    import numpy as np
    from fennol_b200.serving import (ServeRequest, ServeResult, _min_image_ok, atom_steps,
                                     latency_percentiles, serve_requests_from_stream)
    from fennol_b200.systems import request_stream
    assert _min_image_ok(None, 6.2)
    assert _min_image_ok(np.eye(3) * 12.5, 6.2) and not _min_image_ok(np.eye(3) * 12.3, 6.2)
    stream = request_stream(6, seed=1, nmax=60, pool_size=3)
    reqs = serve_requests_from_stream(stream, seed=10)
    assert [q.seed for q in reqs] == list(range(10, 16))
    assert all(q.arrival > 0 for q in reqs)
    res = [ServeResult(q.rid, q.kind, q.natoms, 0.0, None, None, None, 0.0, 0.001 * (k + 1))
           for k, q in enumerate(reqs)]
    lat = latency_percentiles(res)
    assert abs(lat["p50_ms"] - 3.5) < 1e-9
    want = sum(q.natoms * (1 + (q.md_steps if q.kind == "md" else 0)) for q in reqs)
    assert atom_steps(res, {q.rid: q for q in reqs}) == want


def test_aev_active_chunks_cover_every_nonzero_column():
    """For batches with a subset of the species, every non-zero column of the
    oracle's AEV rows lies in a chunk that fennol_aev_active_chunks reports,
    and the mask grows with the species set."""
    from fennol_b200.params import AEVConfig, MLPConfig, init_weights
    from fennol_b200.potential import C_ptr, aev_params
    from fennol_b200.systems import molecule_batch, water_box
    from oracle import ani_ref

    lib = _lib.load()
    cfg = AEVConfig()
    p = aev_params(cfg)
    W = init_weights(cfg, MLPConfig(), seed=0)
    cases = [water_box(3, seed=1)] + molecule_batch(6, seed=12)
    for s in cases:
        cells = None if getattr(s, "cell", None) is None else s.cell[None]
        r = ani_ref.energy_and_forces(s.coordinates, s.species, [s.natoms], W, cfg, MLPConfig(), cells=cells,
                                      need_forces=False, return_aev=True)
        sidx = cfg.species_index(s.species)
        mask = int(np.bitwise_or.reduce(1 << np.unique(sidx)))
        chunks = lib.fennol_aev_active_chunks(C_ptr(p), mask)
        nz = np.nonzero(np.abs(r["aev"]).max(axis=0) > 0)[0]
        assert all((chunks >> (c // 64)) & 1 for c in nz), (mask, bin(chunks))
        assert chunks & ~lib.fennol_aev_active_chunks(C_ptr(p), 0x7F) == 0
    assert lib.fennol_aev_active_chunks(C_ptr(p), 0x7F) == (1 << 16) - 1
