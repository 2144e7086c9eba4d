"""MD controls of the run.in surface, on the GPU through the C ABI and nepx-md.

* correct_velocity N [grouping]: every N steps the driver removes each
  group's linear and angular momentum; checked against a numpy restatement
  of the reference's correct_velocity_subset (src/runtime.cu:979-1063)
  driving the same MD through nepx_md_set_velocity, and against the
  momenta it must remove;
* adaptive time step (time_step dt max_distance): the step size of every
  step is min(dt, max_distance / max|v|) over the velocities at its start
  (reference adaptive_time_step, src/runtime.cu:594-619), and a bound that
  never binds leaves the fixed-step trajectory unchanged bit for bit;
* unwrapped positions (dump_xyz unwrapped_position): the device's running
  sum of displacements against the host's unwrapping of the wrapped path,
  and the column of the nepx-md dump;
* neighbor.out: a record at every 1000th force evaluation, equal to the
  md's own row occupancy of that evaluation.
"""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

import workloads
from conftest import ROOT, potential

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

CLI = os.path.join(ROOT, "dmg-md_b200", "bin", "nepx-md")
WATER = "nep_water.txt"
MASS = {0: 15.999, 1: 1.008}


def _water(n_mol=300, seed=3, T=300.0):
    t, h, p = workloads.water(n_mol=n_mol, seed=seed)
    m = np.array([MASS[int(k)] for k in t])
    v = workloads.maxwell_boltzmann(m, T, seed=seed + 1)
    return t, h, p, m, v


def _md(t, h, p, m, v, kind="nve"):
    import nepx
    pot = nepx.Potential(potential(WATER), max_atoms=len(t))
    md = nepx.MD(pot, t, m, p, v, h)
    md.set_ensemble(kind)
    return pot, md


def _correct(m, pos, vel, idx):
    """The reference's correct_velocity_subset on atoms idx (numpy, FP64)."""
    mm = m[idx]
    M = mm.sum()
    vel[:, idx] -= (vel[:, idx] * mm).sum(axis=1)[:, None] / M
    c = (pos[:, idx] * mm).sum(axis=1) / M
    r = pos[:, idx] - c[:, None]
    L = (mm * np.cross(r.T, vel[:, idx].T).T).sum(axis=1)
    x, y, z = r
    I = np.array([[(mm * (y * y + z * z)).sum(), -(mm * x * y).sum(), -(mm * x * z).sum()],
                  [-(mm * x * y).sum(), (mm * (x * x + z * z)).sum(), -(mm * y * z).sum()],
                  [-(mm * x * z).sum(), -(mm * y * z).sum(), (mm * (x * x + y * y)).sum()]])
    if abs(np.linalg.det(I)) < 1e-10:
        return
    w = np.linalg.solve(I, L)
    vel[:, idx] -= np.cross(w, r.T).T


def _model_xyz(t, h, p, m, v, groups=None):
    sym = {0: "O", 1: "H"}
    H = np.asarray(h).reshape(3, 3)
    lat = " ".join("%.17g" % x for x in H.T.reshape(-1))
    props = "species:S:1:pos:R:3:mass:R:1:vel:R:3" + (":group:I:1" if groups is not None else "")
    lines = ["%d" % len(t), 'pbc="T T T" Lattice="%s" Properties=%s' % (lat, props)]
    for a in range(len(t)):
        row = "%s %.17g %.17g %.17g %.17g %.17g %.17g %.17g" % (
            sym[int(t[a])], p[0, a], p[1, a], p[2, a], m[a], v[0, a], v[1, a], v[2, a])
        if groups is not None:
            row += " %d" % groups[a]
        lines.append(row)
    return "\n".join(lines) + "\n"


def _frames(text, key):
    out, lines, k = [], text.splitlines(), 0
    while k < len(lines):
        n = int(lines[k])
        props = re.search(r"Properties=(\S+)", lines[k + 1]).group(1).split(":")
        col, c = None, 0
        for q in range(0, len(props), 3):
            if props[q] == key:
                col = c
            c += int(props[q + 2])
        rows = np.array([[float(x) for x in lines[k + 2 + a].split()[1:]] for a in range(n)])
        out.append(rows[:, col - 1:col + 2].T)
        k += 2 + n
    return out


@pytest.mark.parametrize("grouped", [False, True])
def test_correct_velocity_matches_restatement(tmp_path, grouped):
    t, h, p, m, v = _water()
    n = len(t)
    groups = (np.arange(n) % 3 == 0).astype(int) if grouped else None
    shutil.copyfile(potential(WATER), tmp_path / "nep.txt")
    (tmp_path / "model.xyz").write_text(_model_xyz(t, h, p, m, v, groups))
    cv = "correct_velocity 10 0" if grouped else "correct_velocity 10"
    (tmp_path / "run.in").write_text("potential nep.txt\ntime_step 0.5\nensemble nve\n%s\n"
                                     "dump_xyz 10 traj.xyz velocity\nrun 30\n" % cv)
    r = subprocess.run([CLI], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    dumped = _frames((tmp_path / "traj.xyz").read_text(), "vel")
    assert len(dumped) == 3
    # the same program through the C ABI, the correction restated in numpy
    sets = [np.nonzero(groups == g)[0] for g in (0, 1)] if grouped else [np.arange(n)]
    pot, md = _md(t, h, p, m, v)
    md.compute_forces()
    for k, done in enumerate((0, 10, 20)):
        st = md.state()
        vel = st["vel"].copy()
        for idx in sets:
            _correct(m, st["pos"], vel, idx)
            # what the correction removes: the group's momentum and angular momentum
            mm = m[idx]
            assert np.abs((vel[:, idx] * mm).sum(axis=1)).max() < 1e-10
            c = (st["pos"][:, idx] * mm).sum(axis=1) / mm.sum()
            Lz = (mm * np.cross((st["pos"][:, idx] - c[:, None]).T, vel[:, idx].T).T).sum(axis=1)
            assert np.abs(Lz).max() < 1e-7
        md.set_velocity(vel)
        md.run_segment(10, 0.5, done, 30)
        got = md.state()["vel"]
        np.testing.assert_allclose(dumped[k], got, rtol=1e-7, atol=1e-10)
    md.close()
    pot.close()


def test_adaptive_time_step():
    t, h, p, m, v = _water(T=600.0)
    pot, md = _md(t, h, p, m, v)
    md.compute_forces()
    dmax = 0.004        # A per step: binds for the fastest hydrogens at dt 0.5 fs
    md.set_max_distance(dmax)
    expected = 0.0
    limited = 0
    for k in range(6):
        st = md.state()
        vmax = np.sqrt((st["vel"] ** 2).sum(axis=0)).max()
        dt = min(0.5, dmax / vmax)
        limited += dt < 0.5
        expected += dt
        md.run_segment(1, 0.5, k, 6)
        assert abs(md.time() - expected) <= 1e-12 * expected, (md.time(), expected)
        # the fastest atom moved about max_distance (its half-kicked speed x dt)
        moved = st["pos"] - md.state()["pos"]
        L = np.diag(np.asarray(h).reshape(3, 3))[:, None]
        moved -= np.round(moved / L) * L
        assert np.sqrt((moved ** 2).sum(axis=0)).max() <= 1.05 * dmax
    assert limited == 6
    md.close()
    # a bound that never binds: the fixed-step trajectory, bit for bit
    runs = []
    for bound in (0.0, 1.0e6):
        pot2, md2 = _md(t, h, p, m, v)
        md2.set_max_distance(bound)
        md2.run(20, 0.5)
        runs.append(md2.state())
        md2.close()
        pot2.close()
    assert np.array_equal(runs[0]["pos"], runs[1]["pos"])
    assert np.array_equal(runs[0]["vel"], runs[1]["vel"])
    pot.close()


def test_unwrapped_positions(tmp_path):
    t, h, p, m, v = _water(T=3000.0)
    L = np.diag(np.asarray(h).reshape(3, 3))[:, None]
    pot, md = _md(t, h, p, m, v)
    md.enable_unwrapped()
    host = md.state()["pos"].copy()
    prev = host.copy()
    for k in range(40):
        md.run_segment(5, 0.5, 5 * k, 200)
        cur = md.state()["pos"]
        d = cur - prev
        host += d - np.round(d / L) * L
        prev = cur
    un = md.unwrapped()
    np.testing.assert_allclose(un, host, rtol=0, atol=1e-9)
    wraps = np.round((un - prev) / L)
    np.testing.assert_allclose(un - prev, wraps * L, rtol=0, atol=1e-9)
    assert np.abs(wraps).max() >= 1                     # some atoms crossed the box
    md.close()
    pot.close()
    # nepx-md writes the column after energy_atom, as the reference does
    shutil.copyfile(potential(WATER), tmp_path / "nep.txt")
    (tmp_path / "model.xyz").write_text(_model_xyz(t, h, p, m, v))
    (tmp_path / "run.in").write_text("potential nep.txt\ntime_step 0.5\nensemble nve\n"
                                     "dump_xyz 100 traj.xyz potential unwrapped_position\n"
                                     "run 200\n")
    r = subprocess.run([CLI], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    text = (tmp_path / "traj.xyz").read_text()
    assert "energy_atom:R:1:unwrapped_position:R:3" in text
    un_cli = _frames(text, "unwrapped_position")[-1]
    pos_cli = _frames(text, "pos")[-1]
    k = np.round((un_cli - pos_cli) / L)
    np.testing.assert_allclose(un_cli - pos_cli, k * L, rtol=0, atol=1e-5)
    assert np.abs(k).max() >= 1


def test_neighbor_out_every_thousand_evaluations(tmp_path):
    t, h, p, m, v = _water()
    shutil.copyfile(potential(WATER), tmp_path / "nep.txt")
    (tmp_path / "model.xyz").write_text(_model_xyz(t, h, p, m, v))
    (tmp_path / "run.in").write_text("potential nep.txt\ntime_step 0.5\nensemble nve\n"
                                     "run 600\nrun 600\n")
    r = subprocess.run([CLI], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = (tmp_path / "neighbor.out").read_text().splitlines()
    # evaluations 0 (first run's initial one) and 1000 (step 398 of the
    # second run: 601 evaluations in the first run, one before the second's steps)
    steps = [int(re.search(r"step (\d+):", x).group(1)) for x in lines]
    assert steps == [0, 1000], lines
    got = [tuple(int(x) for x in re.findall(r"actual=(\d+)", line)) for line in lines]
    pot, md = _md(t, h, p, m, v)
    md.compute_forces()
    want = [md.neighbor_info()]
    md.run_segment(600, 0.5, 0, 600)
    md.compute_forces()
    md.run_segment(399, 0.5, 0, 600)
    want.append(md.neighbor_info())
    assert got == want
    info = pot.info
    assert all("radial(max=%d," % info["MN_r"] in x and "angular(max=%d," % info["MN_a"] in x
               for x in lines)
    md.close()
    pot.close()
