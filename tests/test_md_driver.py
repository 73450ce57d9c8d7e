"""The .fnl input reader of the MD driver (host side)."""

import numpy as np
import pytest

from fennol_b200.md_driver import get, parse_fnl, read_xyz_input

SAMPLE = """
device cuda:0   # comment
matmul_prec highest
model_file model.fnx
xyz_input{
  file box.xyz
  indexed yes
  has_comment_line no
}
cell = 12.0 0. 0. 0. 12.0 0. 0. 0. 12.0
minimum_image yes
nsteps = 40
dt[fs] = .5
nblist_skin 1.
traj_format arc
tdump[ps] = 0.01
nprint = 10
!thermostat NVE
thermostat LGV
temperature = 300.
gamma[THz] = 10.
conservation_tests
"""


def test_parse_sections_units_and_flags():
    p = parse_fnl(SAMPLE)
    assert p["device"] == "cuda:0" and p["matmul_prec"] == "highest"
    assert p["xyz_input"] == {"file": "box.xyz", "indexed": True, "has_comment_line": False}
    assert p["cell"] == [12.0, 0.0, 0.0, 0.0, 12.0, 0.0, 0.0, 0.0, 12.0]
    assert p["nsteps"] == 40 and p["thermostat"] == "LGV" and p["conservation_tests"] is True
    assert get(p, "dt", kind="time") == pytest.approx(0.5e-3)
    assert get(p, "tdump", kind="time") == pytest.approx(0.01)
    assert get(p, "gamma", kind="freq") == pytest.approx(10.0)
    assert get(p, "xyz_input/file") == "box.xyz"
    with pytest.raises(ValueError):
        get(parse_fnl("dt[furlong] = 1"), "dt", kind="time")
    with pytest.raises(ValueError):
        parse_fnl("a{\n b 1\n")


def test_read_tinker_and_plain_xyz(tmp_path):
    (tmp_path / "a.xyz").write_text("3\n1 O 0.0 0.0 0.0 1\n2 H 0.9 0.0 0.0 2\n3 CL 0.0 1.0 0.0 3\n")
    z, x = read_xyz_input(str(tmp_path / "a.xyz"), indexed=True, has_comment_line=False)
    np.testing.assert_array_equal(z, [8, 1, 17])
    np.testing.assert_allclose(x[1], [0.9, 0, 0])
    (tmp_path / "b.xyz").write_text("2\ncomment\nC 0 0 0\nN 1.2 0 0\n")
    z, x = read_xyz_input(str(tmp_path / "b.xyz"), indexed=False, has_comment_line=True)
    np.testing.assert_array_equal(z, [6, 7])
