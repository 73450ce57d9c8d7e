"""Continuous batching: each request's result is the same alone and in the
mix (energies bitwise, forces and MD states to float32 rounding of the
atomic force sums), equal to the direct API, and the MD lane follows the
single-system integrator."""

import numpy as np
import pytest
import torch

from fennol_b200.md import MDEngine
from fennol_b200.params import MD_OUTPUT_SCALE
from fennol_b200.potential import ANIPotential
from fennol_b200.serving import (ServeRequest, ServingEngine, latency_percentiles,
                                 serve_requests_from_stream)
from fennol_b200.systems import molecule_batch, request_stream, water_box

pytestmark = pytest.mark.gpu
F_TOL = 2e-6      # Ha/A (1.3e-3 kcal/mol/A): float32 rounding of atomic force sums
X_TOL = 1e-5      # A after 20 MD steps


@pytest.fixture(scope="module")
def pot(cuda_device):
    return ANIPotential(precision="bf16x2", bf16_weights=True, device=cuda_device,
                        output_scale=MD_OUTPUT_SCALE)


def mixed_requests(md_steps=20):
    mols = molecule_batch(6, seed=21, nmin=8, nmax=60)
    boxes = [water_box(2, seed=1), water_box(3, seed=2), water_box(5, seed=3)]
    reqs = []
    for k, s in enumerate(mols + boxes):
        kind = "md" if k % 3 == 1 else "ef"
        reqs.append(ServeRequest(k, kind, s.species, s.coordinates, s.cell,
                                 md_steps if kind == "md" else 0, None, 100 + k))
    return reqs


def by_rid(results):
    return {r.rid: r for r in results}


def test_alone_equals_mix(pot):
    reqs = mixed_requests()
    mix = by_rid(ServingEngine(pot, segment_steps=10).run(reqs, realtime=False))
    assert len(mix) == len(reqs)
    for q in reqs:
        alone = ServingEngine(pot, segment_steps=10).run([q], realtime=False)[0]
        m = mix[q.rid]
        assert m.kind == alone.kind == q.kind
        if q.kind == "ef":
            assert m.energy == alone.energy, q.rid
            np.testing.assert_allclose(m.forces, alone.forces, rtol=0, atol=F_TOL)
        else:
            np.testing.assert_allclose(m.coordinates, alone.coordinates, rtol=0, atol=X_TOL)
            np.testing.assert_allclose(m.velocities, alone.velocities, rtol=0, atol=1e-2)
            assert abs(m.energy - alone.energy) < 1e-6


def test_single_points_equal_direct_api(pot):
    reqs = [q for q in mixed_requests() if q.kind == "ef"]
    res = by_rid(ServingEngine(pot).run(reqs, realtime=False))
    for q in reqs:
        e, f = pot.energy_and_forces(q.coordinates, q.species, [q.natoms],
                                     None if q.cell is None else q.cell[None])
        assert abs(res[q.rid].energy - float(e[0])) < 1e-9
        np.testing.assert_allclose(res[q.rid].forces, f.cpu().numpy(), rtol=0, atol=F_TOL)


def test_md_lane_follows_md_engine_nve(pot):
    s = water_box(5, seed=8)
    rng = np.random.default_rng(3)
    v0 = rng.standard_normal((s.natoms, 3)) * 5.0
    eng = MDEngine(pot, s.coordinates, s.species, s.cell, thermostat="NVE", velocities=v0, skin=1.0)
    eng.run(20)
    q = ServeRequest(0, "md", s.species, s.coordinates, s.cell, 20, v0, 1)
    r = ServingEngine(pot, thermostat="NVE", segment_steps=10).run([q], realtime=False)[0]
    np.testing.assert_allclose(r.coordinates, eng.x.cpu().numpy(), rtol=0, atol=X_TOL)
    np.testing.assert_allclose(r.velocities, eng.v.cpu().numpy(), rtol=0, atol=1e-2)


def test_tight_budget_still_serves_everything(pot):
    reqs = mixed_requests(md_steps=10)
    eng = ServingEngine(pot, hbm_budget_gb=1e-3, max_ef_atoms=64, max_md_atoms=64, segment_steps=5)
    res = eng.run(reqs, realtime=False)
    assert sorted(r.rid for r in res) == [q.rid for q in reqs]
    assert eng.bytes_in_flight == 0


def test_realtime_stream_latencies(pot):
    stream = request_stream(40, rate_hz=2000.0, seed=5, nmax=400, md_steps=20, pool_size=12)
    reqs = serve_requests_from_stream(stream)
    res = ServingEngine(pot, segment_steps=10).run(reqs, realtime=True)
    assert len(res) == len(reqs)
    lat = latency_percentiles(res)
    assert 0 < lat["p50_ms"] <= lat["p99_ms"]
    assert all(r.done >= r.arrival for r in res)
