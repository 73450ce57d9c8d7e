"""GPU MD: NVE trajectory parity with the float64 oracle integrator, energy
conservation, Langevin temperature, graph replay and overflow rollback."""

import numpy as np
import pytest
import torch

from fennol_b200 import _lib
from fennol_b200.md import KB_KCALMOL, MDEngine, MASS_DA_TO_MD
from fennol_b200.params import ATOMIC_MASSES
from fennol_b200.potential import ANIPotential
from fennol_b200.systems import water_box
from oracle import md_ref

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pot(cuda_device):
    return ANIPotential(precision="fp32", device=cuda_device, seed=0)


@pytest.fixture(scope="module")
def gentle(cuda_device):
    """Random model with a small last layer: stable dynamics (see init_weights)."""
    from fennol_b200.params import MD_OUTPUT_SCALE
    return ANIPotential(precision="fp32", device=cuda_device, seed=0, output_scale=MD_OUTPUT_SCALE)


def test_nve_trajectory_matches_oracle(pot):
    s = water_box(4, seed=21)
    eng = MDEngine(pot, s.coordinates, s.species, s.cell, dt_fs=0.5, thermostat="NVE", skin=1.0, seed=3)
    v0 = eng.v.cpu().numpy().copy()
    eng.run(10, graph_steps=1)
    mass = np.array([ATOMIC_MASSES[int(z)] for z in s.species]) * MASS_DA_TO_MD
    xs, es, _ = md_ref.nve_trajectory(s.coordinates, v0, s.species, [s.natoms], mass, pot.weights,
                                      pot.aev_cfg, pot.mlp_cfg, 0.5e-3, 10, cells=s.cell[None])
    dx = np.abs(eng.x.cpu().numpy() - xs[-1]).max()
    assert dx < 1e-5, dx
    assert abs(eng.potential_energy() - es[-1]) / s.natoms < 1e-4


def test_nve_energy_conservation_and_rebuilds(gentle):
    s = water_box(6, seed=22)
    eng = MDEngine(gentle, s.coordinates, s.species, s.cell, dt_fs=0.5, thermostat="NVE", skin=0.5,
                   temperature=300.0, seed=4, check_every=100)
    e0 = eng.potential_energy() + eng.kinetic_energy()
    eng.run(400, graph_steps=4)
    e1 = eng.potential_energy() + eng.kinetic_energy()
    assert eng.rebuild_count() >= 1          # the displacement trigger fired on the device
    assert abs(e1 - e0) / s.natoms < 3e-3    # kcal/mol/atom over 0.2 ps (no repulsive core)


def test_stride_trigger_matches_displacement_forces(gentle):
    """Both rebuild policies keep the radial list exact, so trajectories agree
    (to float32 summation-order noise: rows are built at different steps)."""
    s = water_box(5, seed=23)
    a = MDEngine(gentle, s.coordinates, s.species, s.cell, thermostat="NVE", skin=1.0, seed=5)
    b = MDEngine(gentle, s.coordinates, s.species, s.cell, thermostat="NVE", skin=1.0, seed=5,
                 trigger="stride", nblist_stride=7)
    a.run(30)
    b.run(30)
    assert np.abs(a.x.cpu().numpy() - b.x.cpu().numpy()).max() < 1e-6


def test_langevin_thermalises(gentle):
    s = water_box(6, seed=24)
    eng = MDEngine(gentle, s.coordinates, s.species, s.cell, thermostat="LGV", gamma_ps=50.0,
                   temperature=300.0, skin=1.0, seed=6)
    temps = []
    for _ in range(10):
        eng.run(50, graph_steps=5)
        temps.append(eng.temperature())
    assert 200.0 < np.mean(temps[3:]) < 400.0
    # noise differs between replays: velocities are not periodic in the replay
    v1 = eng.v.clone()
    eng.run(5, graph_steps=5)
    assert not torch.equal(v1, eng.v)


def test_overflow_rolls_back_and_regrows(gentle):
    s = water_box(6, seed=25)
    eng = MDEngine(gentle, s.coordinates, s.species, s.cell, thermostat="NVE", skin=1.0, seed=7,
                   check_every=10)
    ref = MDEngine(gentle, s.coordinates, s.species, s.cell, thermostat="NVE", skin=1.0, seed=7,
                   check_every=10)
    # shrink the radial capacity below the real row length; the engine must detect,
    # restore, regrow and replay
    from fennol_b200.potential import GraphBuffers
    g = eng.graph_buf
    eng.graph_buf = GraphBuffers(eng.layout, g.cutoff, eng.skin, g.cap, 24)
    eng._graphs.clear()
    eng.flag.fill_(1)  # the first step rebuilds into the undersized buffers inside the graph
    eng.run(20)
    ref.run(20)
    assert eng.graph_buf.cap_r > 24
    assert np.abs(eng.x.cpu().numpy() - ref.x.cpu().numpy()).max() < 1e-6


def test_conditional_rebuild_graph_matches_uncaptured_steps(gentle):
    """Graph-replayed steps hold the displacement rebuild in a conditional node;
    steps launched without capture run the flag-gated rebuild kernels.  Both
    rebuild at the same steps; positions agree to float32 summation-order
    noise (force atomics), which the dynamics amplify over longer runs."""
    s = water_box(6, seed=26)
    a = MDEngine(gentle, s.coordinates, s.species, s.cell, thermostat="NVE", skin=0.2, seed=8,
                 check_every=400)
    b = MDEngine(gentle, s.coordinates, s.species, s.cell, thermostat="NVE", skin=0.2, seed=8,
                 check_every=400)
    r_a0, r_b0 = a.rebuild_count(), b.rebuild_count()
    st = torch.cuda.current_stream().cuda_stream
    # (steps, position tolerance, allowed rebuild-count difference): after 300
    # steps the grown noise may move one trigger by a step
    for steps, tol, drb in ((30, 1e-6, 0), (270, 1e-3, 1)):
        a.run(steps, graph_steps=3)
        for _ in range(steps):
            b._launch_step(st, None)
        torch.cuda.synchronize()
        assert a.pot.check_status(a.ws, a.graph_buf) is None
        assert b.pot.check_status(b.ws, b.graph_buf) is None
        ra, rb = a.rebuild_count() - r_a0, b.rebuild_count() - r_b0
        assert ra >= 1 and abs(ra - rb) <= drb
        assert np.abs(a.x.cpu().numpy() - b.x.cpu().numpy()).max() < tol


def test_checked_stride_rolls_back_a_too_long_stride(gentle):
    """Stride mode checks every step's displacement on the device: a stride far
    too long for the skin is caught, the chunk replayed with shorter strides,
    and the trajectory matches the displacement-triggered one."""
    s = water_box(5, seed=27)
    a = MDEngine(gentle, s.coordinates, s.species, s.cell, thermostat="NVE", skin=0.3, seed=9,
                 trigger="stride", nblist_stride=500, check_every=20)
    b = MDEngine(gentle, s.coordinates, s.species, s.cell, thermostat="NVE", skin=0.3, seed=9,
                 check_every=20)
    a.run(40)
    b.run(40)
    assert a.stride_reductions >= 1 and a.nblist_stride < 500
    assert not a.displaced_beyond_skin()
    assert np.abs(a.x.cpu().numpy() - b.x.cpu().numpy()).max() < 1e-5
