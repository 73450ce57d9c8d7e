"""The .fnl MD driver end to end on the GPU: input file, model file, frames,
printed energies and the restart file."""

import io

import numpy as np
import pytest

from fennol_b200.md_driver import parse_fnl, run
from fennol_b200.systems import water_box
from fennol_b200.trajectory import load_restart, read_xyz

pytestmark = pytest.mark.gpu


def write_box(path, s):
    sym = {1: "H", 8: "O"}
    lines = [str(s.natoms)] + [f"{k + 1} {sym[int(z)]} {x:.6f} {y:.6f} {w:.6f} 1"
                               for k, (z, (x, y, w)) in enumerate(zip(s.species, s.coordinates))]
    path.write_text("\n".join(lines) + "\n")


def test_driver_random_model(tmp_path, cuda_device):
    s = water_box(5, seed=1)
    write_box(tmp_path / "box.xyz", s)
    L = s.cell[0, 0]
    text = f"""
precision bf16x2
random_model_seed 3
xyz_input{{
  file box.xyz
  indexed yes
  has_comment_line no
}}
cell = {L} 0 0 0 {L} 0 0 0 {L}
minimum_image yes
nsteps 40
dt[fs] = 0.5
nblist_skin 1.0
traj_format xyz
tdump[fs] = 5
nprint 10
thermostat LGV
temperature 300
gamma[THz] 1
"""
    out = io.StringIO()
    eng = run(parse_fnl(text), tmp_path, out=out)
    rows = [ln.split() for ln in out.getvalue().splitlines() if ln and not ln.startswith("#")]
    assert [int(r[0]) for r in rows] == [10, 20, 30, 40]
    assert all(np.isfinite(float(r[4])) for r in rows)
    frames = read_xyz(str(tmp_path / "box.traj.xyz"))
    assert len(frames) == 4
    np.testing.assert_allclose(frames[-1][1], eng.x.cpu().numpy(), rtol=1e-5, atol=1e-4)
    d = load_restart(str(tmp_path / "box.dyn.restart"), species=s.species)
    assert abs(d["simulation_time_ps"] - 0.02) < 1e-12


def test_driver_model_file(tmp_path, cuda_device):
    from collections import OrderedDict
    from fennol_b200.fennix import FENNIX
    from test_fennix_api import ani_modules, ani_preprocessing

    m = FENNIX(5.2, ani_modules(), ani_preprocessing(), energy_terms=["energy"], rng_key=2)
    m.save(tmp_path / "model.fnx")
    s = water_box(4, seed=2)
    write_box(tmp_path / "box.xyz", s)
    L = s.cell[0, 0]
    text = f"""
model_file model.fnx
matmul_prec highest
xyz_input{{
  file box.xyz
  indexed yes
  has_comment_line no
}}
cell {L} 0 0 0 {L} 0 0 0 {L}
nsteps 4
dt[fs] 0.1
thermostat NVE
nprint 2
"""
    out = io.StringIO()
    run(parse_fnl(text), tmp_path, out=out)
    rows = [ln.split() for ln in out.getvalue().splitlines() if ln and not ln.startswith("#")]
    assert [int(r[0]) for r in rows] == [2, 4]
