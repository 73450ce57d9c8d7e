"""Trajectory formats and restart files (host side)."""

import numpy as np
import pytest

from fennol_b200.trajectory import (cell_lengths_angles, format_frame, load_restart, read_xyz,
                                    save_restart, symbols_of)


def test_cell_lengths_angles():
    np.testing.assert_allclose(cell_lengths_angles(np.diag([10.0, 12.0, 14.0])), [10, 12, 14, 90, 90, 90])
    tri = np.array([[10.0, 0, 0], [5.0, 8.660254037844387, 0], [0, 0, 9.0]])
    np.testing.assert_allclose(cell_lengths_angles(tri), [10, 10, 9, 90, 90, 60], atol=1e-9)


@pytest.mark.parametrize("fmt", ["xyz", "extxyz"])
def test_xyz_round_trip(tmp_path, fmt):
    rng = np.random.default_rng(0)
    x = rng.normal(size=(5, 3)) * 3
    sym = symbols_of([8, 1, 1, 6, 17])
    f = rng.normal(size=(5, 3))
    path = tmp_path / "t.xyz"
    with open(path, "w") as fh:
        for k in range(3):
            fh.write(format_frame(fmt, sym, x + k, cell=np.eye(3) * 20.0,
                                  forces=f if fmt == "extxyz" else None, properties={"step": k}))
    frames = read_xyz(str(path))
    assert len(frames) == 3
    for k, (s, xr, comment) in enumerate(frames):
        assert s == ["O", "H", "H", "C", "Cl"]
        np.testing.assert_allclose(xr, x + k, rtol=1e-5, atol=1e-5)
        if fmt == "extxyz":
            assert 'Lattice="20.000' in comment and ":forces:R:3" in comment and f"step={k}" in comment
        else:
            assert comment.split() == ["20.000", "20.000", "20.000", "90.000", "90.000", "90.000"]


def test_arc_frame_layout():
    txt = format_frame("arc", ["O", "H"], np.array([[0.0, 1.0, 2.0], [3.0, 4.0, 5.0]]), cell=np.eye(3) * 9)
    lines = txt.splitlines()
    assert lines[0] == "2" and lines[1].split()[:3] == ["9.00000", "9.00000", "9.00000"]
    assert lines[2].split() == ["1", "O", "0.000", "1.000", "2.000"]
    assert lines[3].split()[0:2] == ["2", "H"]


def test_restart_round_trip(tmp_path):
    sp = np.array([8, 1, 1])
    x, v = np.arange(9.0).reshape(3, 3), -np.arange(9.0).reshape(3, 3)
    save_restart(str(tmp_path / "r.pkl"), sp, x, v, 1.5, cell=np.eye(3) * 10)
    d = load_restart(str(tmp_path / "r.pkl"), species=sp)
    assert d["nat"] == 3 and d["simulation_time_ps"] == 1.5 and d["cells"].shape == (1, 3, 3)
    np.testing.assert_array_equal(d["coordinates"], x)
    np.testing.assert_array_equal(d["vel"], v)
    with pytest.raises(ValueError):
        load_restart(str(tmp_path / "r.pkl"), species=np.array([8, 1, 6]))
