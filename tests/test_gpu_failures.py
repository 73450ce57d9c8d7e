"""Failure detection on the GPU without a GPU fault: non-finite values found by
the device check (FeNNol's MD driver raises on NaN positions or velocities,
md/dynamic.py:204-208, 595-597), and a bounded wait of the fused tensor-core
MLP that runs out (the load producer is told to issue nothing, so no copy is
in flight) with the context usable afterwards."""

import numpy as np
import pytest
import torch

from fennol_b200 import _lib
from fennol_b200.md import MDEngine
from fennol_b200.params import MD_OUTPUT_SCALE
from fennol_b200.potential import ANIPotential
from fennol_b200.serving import ServeRequest, ServingEngine
from fennol_b200.systems import water_box

pytestmark = pytest.mark.gpu


def test_nan_in_host_coordinates_is_refused_before_upload(cuda_device):
    pot = ANIPotential(precision="fp32", device=cuda_device, seed=0)
    s = water_box(4, seed=0)
    x = s.coordinates.copy()
    x[7, 1] = np.nan
    with pytest.raises(ValueError, match="NaN"):
        pot.energy_and_forces(x, s.species, [s.natoms], s.cell[None])
    with pytest.raises(ValueError, match="NaN"):
        MDEngine(pot, x, s.species, s.cell)


@pytest.mark.parametrize("precision", ["fp32", "f16x3x1"])
def test_nan_in_device_coordinates_sets_the_status_word(cuda_device, precision):
    """An atom at a NaN position drops out of every neighbour list (its
    distances fail the cutoff test), so the energy alone can stay finite; the
    device check of the positions reports it."""
    pot = ANIPotential(precision=precision, device=cuda_device, seed=0)
    s = water_box(4, seed=0)
    x = torch.tensor(s.coordinates, dtype=torch.float32, device=cuda_device)
    e, _ = pot.energy_and_forces(x, s.species, [s.natoms], s.cell[None])
    assert torch.isfinite(e).all()
    x[11, 2] = float("inf")
    with pytest.raises(_lib.NonFiniteError):
        pot.energy_and_forces(x, s.species, [s.natoms], s.cell[None])
    x[11, 2] = float(s.coordinates[11, 2])
    e2, _ = pot.energy_and_forces(x, s.species, [s.natoms], s.cell[None])
    assert abs(float(e2[0]) - float(e[0])) < 1e-9


def test_md_raises_when_positions_turn_nan(cuda_device):
    pot = ANIPotential(precision="f16x3x1", device=cuda_device, seed=0, output_scale=MD_OUTPUT_SCALE)
    s = water_box(4, seed=1)
    eng = MDEngine(pot, s.coordinates, s.species, s.cell, dt_fs=0.5, thermostat="NVE", skin=1.0)
    eng.run(10)
    eng.v[3, 0] = float("nan")   # written from the host between chunks
    with pytest.raises(ValueError, match="dynamics crashed"):
        eng.run(10)


def test_serving_refuses_a_nan_request_and_serves_the_others(cuda_device):
    pot = ANIPotential(precision="f16x3x1", device=cuda_device, seed=0, output_scale=MD_OUTPUT_SCALE)
    s = water_box(3, seed=2)
    bad = s.coordinates.copy()
    bad[0, 0] = np.nan
    reqs = [ServeRequest(0, "ef", s.species, s.coordinates, s.cell),
            ServeRequest(1, "ef", s.species, bad, s.cell),
            ServeRequest(2, "ef", s.species, s.coordinates + 0.01, s.cell)]
    res = {r.rid: r for r in ServingEngine(pot).run(reqs, realtime=False)}
    assert res[1].error is not None and res[0].error is None and res[2].error is None
    assert np.isfinite(res[0].energy) and np.isfinite(res[2].energy)


def test_mlp_wait_timeout_sets_error_and_context_recovers(cuda_device):
    """The next fused launch starts with a producer that issues no loads: the
    MMA and epilogue waits run out after a short limit, the error word is
    set (raised as KernelTimeout), the kernel frees its tensor memory and
    returns, and the next normal call gives the same result as before."""
    lib = _lib.load()
    pot = ANIPotential(precision="f16x3x1", device=cuda_device, seed=0)
    s = water_box(4, seed=3)
    e0, f0 = pot.energy_and_forces(s.coordinates, s.species, [s.natoms], s.cell[None])
    e0, f0 = float(e0[0]), f0.cpu().numpy().copy()
    assert lib.fennol_mlp_wait_limit(0.05) == 0
    assert lib.fennol_mlp_inject_stall(1) == 0
    try:
        with pytest.raises(_lib.KernelTimeout):
            pot.energy_and_forces(s.coordinates + 1e-3, s.species, [s.natoms], s.cell[None])
    finally:
        lib.fennol_mlp_inject_stall(0)
        lib.fennol_mlp_wait_limit(2.0)
    torch.cuda.synchronize()
    e1, f1 = pot.energy_and_forces(s.coordinates, s.species, [s.natoms], s.cell[None])
    assert abs(float(e1[0]) - e0) < 1e-9
    np.testing.assert_allclose(f1.cpu().numpy(), f0, rtol=0, atol=1e-6)
    assert lib.fennol_mlp_wait_limit(0.0) == _lib.ERR_INVALID
    assert lib.fennol_mlp_inject_stall(-1) == _lib.ERR_INVALID
