"""GPU tests of the device-resident MD loop (nepx_md_* through the C ABI)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import workloads
from conftest import ROOT, potential

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

K_B = 8.617343e-5
MASS_C = 12.011


def _nepx():
    import nepx
    return nepx


def test_nve_follows_gpumd_golden_trajectory(goldens):
    """6 NVE steps of 0.1 fs from the reference suite's single_large_nve case.

    Positions at the suite's tolerance (rtol 2e-8, atol 2e-9 A); velocities at
    5x the suite's (the FP32 force rounding differs from GPUMD's by ~5e-6 eV/A,
    which alone moves v by ~2.5e-9 A/fs over 0.6 fs); forces, per-atom
    energies and virials at the suite's force/energy/virial tolerances.
    """
    nepx = _nepx()
    tr = goldens["trajectories"]["single_large_nve"]
    model = tr["model"]
    n = model["n"]
    pot = nepx.Potential(potential(tr["potential"]), max_atoms=n)
    md = nepx.MD(pot, model["type"], [MASS_C] * n, np.array(model["pos"]).T,
                 np.array(model["vel"]).T, model["h"])
    md.set_ensemble("nve")
    rowmajor = [0, 3, 4, 6, 1, 5, 7, 8, 2]
    for frame in tr["frames"]:
        md.run(1, 0.1)
        s = md.state()
        pos = np.array(frame["pos"]).T
        vel = np.array(frame["vel"]).T
        assert np.all(np.abs(s["pos"] - pos) <= 2e-9 + 2e-8 * np.abs(pos)), frame["time_fs"]
        assert np.all(np.abs(s["vel"] - vel) <= 5 * (2e-9 + 2e-7 * np.abs(vel))), frame["time_fs"]
        f = np.array(frame["force"]).T
        assert np.all(np.abs(s["force"] - f) <= 1e-6 + 1e-4 * np.abs(f) + 1e-5)
        e = np.array(frame["energy_atom"])
        assert np.all(np.abs(s["pe"] - e) <= 2e-5 + 1e-5 * np.abs(e))
        w = np.array(frame["virial_rowmajor"]).T
        assert np.all(np.abs(s["virial"][rowmajor] - w) <= 1e-5 + 1e-4 * np.abs(w))


def _water_md(n_mol, T, struct_seed, kind="nve", **ens):
    nepx = _nepx()
    t, h, p = workloads.water(n_mol=n_mol, seed=struct_seed)
    masses = np.where(t == 0, 15.999, 1.008)
    v = workloads.maxwell_boltzmann(masses, T, seed=struct_seed)
    pot = nepx.Potential(potential("nep_water.txt"), max_atoms=len(t))
    md = nepx.MD(pot, t, masses, p, v, h)
    md.set_ensemble(kind, **ens)
    return pot, md, t, h


def test_nve_energy_conservation():
    """Diamond carbon with the reference's carbon NEP, NVE at dt 0.5 fs.

    The total energy per atom stays within 2e-4 eV of its mean and
    drifts by less than 0.05 eV/atom/ns (the dt^2 integration error of this
    stiff model at ~800 K dominates; halving dt quarters it)."""
    nepx = _nepx()
    t, h, p = workloads.diamond(ncell=6, jitter=0.05, seed=1)
    masses = np.full(len(t), MASS_C)
    v = workloads.maxwell_boltzmann(masses, 300.0, seed=3)
    pot = nepx.Potential(potential("nep_C.txt"), max_atoms=len(t))
    md = nepx.MD(pot, t, masses, p, v, h)
    md.set_ensemble("nve")
    rows = md.run(1000, 0.5, thermo_every=20)
    etot = (rows[:, 1] + rows[:, 2]) / len(t)
    time_ns = np.arange(1, len(rows) + 1) * 20 * 0.5e-6
    slope = np.polyfit(time_ns[5:], etot[5:], 1)[0]
    assert abs(slope) < 0.05, "drift %g eV/atom/ns" % slope
    assert np.abs(etot[5:] - etot[5:].mean()).max() < 2e-4


def test_bdp_velocity_factor_bit_exact(tmp_path):
    """Device resampling equals the reference formula on the same draws."""
    lib = tmp_path / "libsvr.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off",
                    os.path.join(ROOT, "tests", "cpp", "svr_harness.cpp"), "-o", str(lib)],
                   check=True)
    L = ctypes.CDLL(str(lib))
    dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
    L.svr_step_draws.argtypes = [ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]
    L.resample.restype = ctypes.c_double
    L.resample.argtypes = [ctypes.c_double] * 2 + [ctypes.c_int] + [ctypes.c_double] * 3
    steps, seed = 60, 2024
    pot, md, t, h = _water_md(200, 250.0, 2, kind="nvt_bdp", T0=300.0, T1=320.0, Tdamp=20.0,
                              seed=seed)
    rows = md.run(steps, 0.5, thermo_every=1)
    n = len(t)
    ndeg = 3 * n
    draws = np.zeros(3 * steps)
    L.svr_step_draws(seed, ndeg, steps, 0, draws)
    factor = np.exp(-1.0 / 20.0)
    for k in range(steps):
        T = rows[k, 0]
        Tt = 300.0 + (320.0 - 300.0) * (float(k) / float(steps))
        old = T * ndeg * K_B * 0.5
        sigma = ndeg * K_B * Tt * 0.5
        new = L.resample(old, sigma, ndeg, factor, draws[3 * k], draws[3 * k + 1])
        assert np.sqrt(new / old) == rows[k, 18], k


@pytest.mark.parametrize("kind,ens", [("nvt_bdp", dict(T0=300.0, T1=330.0, Tdamp=20.0)),
                                      ("nvt_nhc", dict(T0=300.0, T1=300.0, Tdamp=50.0)),
                                      ("npt_scr", dict(T0=300.0, T1=300.0, Tdamp=50.0,
                                                       p_gpa=0.0, bulk_gpa=2.0, tau_p=500.0))])
def test_one_step_calls_equal_one_run(kind, ens):
    """A segment driven one step per call (each call one graph: the draws'
    upload, the segment bookkeeping, the step and the status readback) is the
    same trajectory, bit for bit, as the segment run in a single call."""
    steps = 24
    out = []
    for per_step in (False, True):
        pot, md, t, h = _water_md(150, 300.0, 9, kind=kind, seed=77, **ens)
        if per_step:
            rows = np.concatenate([md.run_segment(1, 0.5, k, steps, thermo_every=1)
                                   for k in range(steps)])
        else:
            rows = md.run_segment(steps, 0.5, 0, steps, thermo_every=1)
        s = md.state()
        out.append((rows, s["pos"], s["vel"], s["h"]))
        md.close()
        pot.close()
    (r0, p0, v0, h0), (r1, p1, v1, h1) = out
    assert r0.shape == (steps, 20) and np.isfinite(r0).all()
    assert np.array_equal(r0, r1)
    assert np.array_equal(p0, p1) and np.array_equal(v0, v1) and np.array_equal(h0, h1)


def test_buffers_regrow_inside_a_segment():
    """Calls of 1, 9 and 20 steps inside one 30-step segment: the draw and
    row buffers grow between calls while the step parameters stay the same,
    so the captured graphs must follow the new buffers.  The trajectory is
    the one-call segment's, bit for bit, and a second MD on the same handle
    afterwards runs cleanly."""
    ens = dict(T0=300.0, T1=320.0, Tdamp=20.0, seed=5)
    out = []
    for calls in ([30], [1, 9, 20]):
        pot, md, t, h = _water_md(150, 300.0, 12, kind="nvt_bdp", **ens)
        rows, first = [], 0
        for c in calls:
            rows.append(md.run_segment(c, 0.5, first, 30, thermo_every=1))
            first += c
        s = md.state()
        out.append((np.concatenate(rows), s["pos"], s["vel"]))
        md.close()
        md2 = _nepx().MD(pot, t, np.where(t == 0, 15.999, 1.008), s["pos"], s["vel"], h)
        md2.set_ensemble("nve")
        r2 = md2.run(4, 0.5, thermo_every=2)
        assert np.isfinite(r2).all()
        md2.close()
        pot.close()
    (r0, p0, v0), (r1, p1, v1) = out
    assert r0.shape == (30, 20)
    assert np.array_equal(r0, r1)
    assert np.array_equal(p0, p1) and np.array_equal(v0, v1)


@pytest.mark.parametrize("kind", ["nvt_ber", "nvt_nhc", "nvt_bdp"])
def test_thermostats_reach_target(kind):
    """Diamond carbon started at 200 K is driven to 500 K (Tdamp 50 steps)."""
    nepx = _nepx()
    t, h, p = workloads.diamond(ncell=6, jitter=0.0, seed=5)
    masses = np.full(len(t), MASS_C)
    v = workloads.maxwell_boltzmann(masses, 200.0, seed=5)
    pot = nepx.Potential(potential("nep_C.txt"), max_atoms=len(t))
    md = nepx.MD(pot, t, masses, p, v, h)
    md.set_ensemble(kind, T0=500.0, T1=500.0, Tdamp=20.0)
    rows = md.run(4000, 1.0, thermo_every=10)
    T_late = rows[-200:, 0].mean()   # a Nose-Hoover chain oscillates about the target
    assert abs(T_late - 500.0) < 0.1 * 500.0, (kind, T_late)


@pytest.mark.parametrize("kind", ["npt_ber", "npt_scr"])
def test_npt_box_moves_and_lists_stay_complete(kind):
    nepx = _nepx()
    pot, md, t, h = _water_md(300, 300.0, 4, kind=kind, T0=300.0, Tdamp=20.0, p_gpa=0.5,
                              bulk_gpa=2.0, tau_p=50.0)
    rows = md.run(300, 0.5, thermo_every=10)
    assert np.all(rows[:, 19] > 0)
    assert abs(rows[-1, 9] - h[0]) > 1e-4          # the box moved
    # Berendsen factor = 1 - pc (P_target - P_inst)
    if kind == "npt_ber":
        pc = 1.0 / (3.0 * 50.0 * 2.0)
        p_inst = rows[:, 3:6].mean(axis=1)
        np.testing.assert_allclose(rows[:, 19], 1.0 - pc * (0.5 - p_inst), rtol=0, atol=1e-12)
    # the Verlet list kept across box rescalings must yield exactly the
    # typewise rows a freshly built list yields at the same positions and box;
    # forces then agree to rounding (the lane that sums a radial edge follows
    # its slot in the Verlet row, which differs between the two lists)
    md.set_ensemble("nve")
    md.run(1, 0.0)
    md.sync()
    s = md.state()
    kept = [pot.neighbors(w, len(t)) for w in (0, 1)]
    tt = torch.as_tensor(t, device="cuda")
    pp = torch.as_tensor(np.ascontiguousarray(s["pos"]), device="cuda")
    pot.notify_box_changed()
    pe, f, w = pot.compute(tt, s["h"], pp, sync_check=True)
    fresh = [pot.neighbors(w_, len(t)) for w_ in (0, 1)]
    for a, b in zip(kept, fresh):
        for i in range(len(t)):
            assert np.array_equal(a[i], b[i]), i
    f = f.cpu().numpy()
    assert np.linalg.norm(f - s["force"]) / np.linalg.norm(f) < 1e-6
    assert np.abs(pe.cpu().numpy() - s["pe"]).max() < 1e-5
