"""Trajectory frames streamed off the device during MD, and restarts."""

import numpy as np
import pytest

from fennol_b200.md import MDEngine
from fennol_b200.params import MD_OUTPUT_SCALE
from fennol_b200.potential import ANIPotential
from fennol_b200.systems import water_box
from fennol_b200.trajectory import FrameStream, load_restart, read_xyz

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pot(cuda_device):
    return ANIPotential(precision="bf16x2", bf16_weights=True, device=cuda_device, output_scale=MD_OUTPUT_SCALE)


def test_frames_follow_the_run(pot, tmp_path):
    s = water_box(5, seed=2)
    eng = MDEngine(pot, s.coordinates, s.species, s.cell, thermostat="NVE", seed=1)
    ref = MDEngine(pot, s.coordinates, s.species, s.cell, thermostat="NVE", seed=1)
    fs = FrameStream(str(tmp_path / "t.xyz"), s.species, "xyz", cell=s.cell)
    eng.run_with_frames(20, 5, fs)
    fs.close()
    frames = read_xyz(str(tmp_path / "t.xyz"))
    assert len(frames) == 4
    for k in range(4):
        ref.run(5)
        np.testing.assert_allclose(frames[k][1], ref.x.cpu().numpy(), rtol=1e-5, atol=1e-4)
    np.testing.assert_allclose(frames[-1][1], eng.x.cpu().numpy(), rtol=1e-5, atol=1e-5)


def test_restart_continues_the_trajectory(pot, tmp_path):
    s = water_box(5, seed=3)
    a = MDEngine(pot, s.coordinates, s.species, s.cell, thermostat="NVE", seed=4)
    a.run(10)
    a.save_restart(str(tmp_path / "r.pkl"))
    d = load_restart(str(tmp_path / "r.pkl"), species=s.species)
    assert abs(d["simulation_time_ps"] - 10 * a.dt) < 1e-12
    b = MDEngine(pot, d["coordinates"], d["species"], d["cells"][0], thermostat="NVE",
                 velocities=d["vel"])
    a.run(10)
    b.run(10)
    np.testing.assert_allclose(b.x.cpu().numpy(), a.x.cpu().numpy(), rtol=0, atol=1e-5)
