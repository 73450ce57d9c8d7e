"""The allocation-free neighbour search against the workspace entry point.

``fennol_graph_build_noalloc`` exists for callers that cannot allocate device
memory: an XLA FFI handler (the framework owns every buffer, so the call may
not create memory of its own) or a stream under CUDA graph capture (where
cudaMalloc is not allowed).  Its cell-list scratch is a fixed array inside the
library.  This test calls it through the C ABI twice in a row, with different
coordinates each time, and checks each result against ``fennol_graph_build``
with a caller workspace.  Neighbour rows are integer data, so the comparison
is exact.  The file name sorts last so that a stopping run has already run
every other test.
"""

import ctypes as C

import numpy as np
import pytest
import torch

from fennol_b200 import _lib
from fennol_b200.potential import ANIPotential, GraphBuffers
from fennol_b200.systems import water_box

pytestmark = pytest.mark.gpu

CUTOFF = 5.2


def _rows(nj, ns, nn):
    nn = nn.cpu().numpy()
    nj = nj.cpu().numpy()
    ns = ns.cpu().numpy()
    return nn, [(nj[i, :nn[i]].copy(), ns[i, :nn[i]].copy()) for i in range(nn.shape[0])]


def _noalloc_call(layout, g, coords, nbr_j, nbr_s, nbr_n, status, stream):
    lib = _lib.load()
    return lib.fennol_graph_build_noalloc(
        coords.data_ptr(), layout.n, layout.t_atom_sys.data_ptr(), layout.nsys,
        layout.t_sys_start.data_ptr(), layout.t_mode.data_ptr(), layout.t_cell.data_ptr(),
        layout.t_recip.data_ptr(), g.grid.data_ptr(), g.nrep.data_ptr(), g.ncells, CUTOFF, g.cap,
        nbr_j.data_ptr(), nbr_s.data_ptr(), nbr_n.data_ptr(), status.data_ptr(), None, stream)


def test_noalloc_matches_workspace_entry_point_twice(cuda_device):
    pot = ANIPotential(precision="fp32", device=cuda_device)
    lib = _lib.load()
    max_atoms, max_cells, scratch = C.c_int(), C.c_int(), C.c_size_t()
    assert lib.fennol_graph_noalloc_limits(C.byref(max_atoms), C.byref(max_cells), C.byref(scratch)) == 0
    stream = torch.cuda.current_stream().cuda_stream

    box = water_box(10, seed=31)                      # 3000 atoms, cell-list path
    layout = pot.layout(box.species, [box.natoms], box.cell[None])
    assert layout.n <= max_atoms.value
    ref = GraphBuffers(layout, CUTOFF, 0.0, 96, 96)
    assert 0 < ref.ncells <= max_cells.value
    out_j = torch.full_like(ref.nbr_j, -7)
    out_s = torch.full_like(ref.nbr_s, -7)
    out_n = torch.full_like(ref.nbr_n, -7)
    st_ref = torch.zeros(_lib.STATUS_WORDS, dtype=torch.int32, device=cuda_device)
    st_new = torch.zeros_like(st_ref)

    rng = np.random.default_rng(5)
    positions = [box.coordinates, box.coordinates + rng.uniform(-0.3, 0.3, box.coordinates.shape)]
    for x in positions:  # two calls in a row; the second reuses the shared scratch
        coords = torch.tensor(x, dtype=torch.float32, device=cuda_device)
        st_ref.zero_()
        st_new.zero_()
        ref.build(layout, coords, st_ref, stream)
        rc = _noalloc_call(layout, ref, coords, out_j, out_s, out_n, st_new, stream)
        assert rc == _lib.OK
        torch.cuda.synchronize()
        assert int(st_ref[_lib.ST_NBR_OVERFLOW]) == 0
        assert torch.equal(st_ref, st_new)
        n_ref, rows_ref = _rows(ref.nbr_j, ref.nbr_s, ref.nbr_n)
        n_new, rows_new = _rows(out_j, out_s, out_n)
        assert np.array_equal(n_ref, n_new)
        for (a, b), (c, d) in zip(rows_ref, rows_new):
            assert np.array_equal(a, c) and np.array_equal(b, d)


def test_noalloc_rejects_inputs_beyond_its_scratch(cuda_device):
    lib = _lib.load()
    max_atoms = C.c_int()
    lib.fennol_graph_noalloc_limits(C.byref(max_atoms), None, None)
    rc = lib.fennol_graph_build_noalloc(None, max_atoms.value + 1, None, 1, None, None, None, None, None,
                                        None, 0, CUTOFF, 64, None, None, None, None, None, None)
    assert rc == _lib.ERR_STATIC_LIMIT
