"""Print-state files and the reference's comparison (CompareStateFiles) on
the CPU: Java time strings, a round trip, known errors for particles and
frames, and the consistency checks the reference makes."""
import io
import math

import numpy as np
import pytest

from artisynth_core_b200 import statefile as S


def test_java_double_strings():
    cases = {0.0: "0.0", 0.01: "0.01", 1.0: "1.0", 0.005: "0.005", 123.25: "123.25", 1e-4: "1.0E-4",
             1.5e7: "1.5E7", 0.3: "0.3", 2.5e-5: "2.5E-5", 1e7: "1.0E7"}
    for d, s in cases.items():
        assert S.java_double(d) == s, (d, S.java_double(d))


def _write(path, comps, times, vel, pos, fmt="%.17g", desc="beam"):
    w = S.StateWriter(str(path), fmt=fmt)
    w.header(desc, comps)
    for t, v, x in zip(times, vel, pos):
        w.state(t, v, x)
    w.close()


def _traj(seed, n_t=4):
    rng = np.random.default_rng(seed)
    comps = ["P", "P", "F", "R2", "P"]
    nv, nx = 3 + 3 + 6 + 2 + 3, 3 + 3 + 7 + 2 + 3
    vel = [rng.standard_normal(nv) for _ in range(n_t)]
    pos = []
    for _ in range(n_t):
        x = rng.standard_normal(nx)
        q = rng.standard_normal(4)
        x[6:10] = q / np.linalg.norm(q)
        pos.append(x)
    return comps, [0.01 * k for k in range(n_t)], vel, pos


def test_round_trip_compares_equal(tmp_path):
    comps, times, vel, pos = _traj(1)
    _write(tmp_path / "a.out", comps, times, vel, pos)
    secs = S.read_file(str(tmp_path / "a.out"))
    assert len(secs) == 1 and secs[0].comps == comps and secs[0].times == times
    assert all(np.array_equal(a, b) for a, b in zip(secs[0].vel, vel))
    out = io.StringIO()
    assert S.compare_files(str(tmp_path / "a.out"), str(tmp_path / "a.out"), out=out) == (0.0, 0.0)
    assert "max vel error=0 at" in out.getvalue()


def test_particle_error_is_normalised_by_largest_magnitude(tmp_path):
    comps = ["P", "P"]
    v = [np.array([1.0, 0, 0, 0, 3.0, 4.0])]
    x = [np.array([0.0, 0, 0, 1, 1, 1])]
    v2 = [v[0].copy()]
    v2[0][0] += 0.5  # particle 0 velocity off by 0.5
    x2 = [x[0].copy()]
    x2[0][3:6] += 0.1  # particle 1 position off by 0.1 * sqrt(3)
    _write(tmp_path / "a", comps, [0.0], v, x)
    _write(tmp_path / "b", comps, [0.0], v2, x2)
    ve, pe = S.compare_files(str(tmp_path / "a"), str(tmp_path / "b"), show_level=-1)
    # largest velocity magnitude: particle 1, |(0, 3, 4)| = 5
    assert ve == pytest.approx(0.5 / 5.0)
    assert pe == pytest.approx(0.1 * math.sqrt(3) / np.linalg.norm([1.1, 1.1, 1.1]))


def test_frame_orientation_error_is_angle_over_pi(tmp_path):
    comps = ["F"]
    th = 0.3
    q1 = np.array([1.0, 0, 0, 0])
    q2 = np.array([math.cos(th / 2), 0, 0, math.sin(th / 2)])
    v = [np.zeros(6)]
    _write(tmp_path / "a", comps, [0.0], v, [np.concatenate([[1, 2, 3], q1])])
    _write(tmp_path / "b", comps, [0.0], v, [np.concatenate([[1, 2, 3], q2])])
    _, pe = S.compare_files(str(tmp_path / "a"), str(tmp_path / "b"), show_level=-1)
    assert pe == pytest.approx(th / math.pi)


def test_inconsistent_files_are_rejected(tmp_path):
    comps, times, vel, pos = _traj(2)
    _write(tmp_path / "a", comps, times, vel, pos)
    _write(tmp_path / "b", comps, times, vel, pos, desc="other")
    with pytest.raises(ValueError):
        S.compare_files(str(tmp_path / "a"), str(tmp_path / "b"), show_level=-1)
    _write(tmp_path / "c", comps, [t + 1 for t in times], vel, pos)
    with pytest.raises(ValueError):
        S.compare_files(str(tmp_path / "a"), str(tmp_path / "c"), show_level=-1)
