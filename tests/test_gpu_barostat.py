"""Anisotropic and triclinic pressure coupling (nepx_md_set_barostat).

The reference has only the isotropic barostat and rejects the others
(src/box_control.cpp:14-23); these couplings follow GPUMD's per-component
form.  The tests restate the box update on the host from the engine's own
thermo rows, which carry each step's pressure tensor (GPa) and the box after
that step's update:
  mu_aa = 1 - (P0_a - P_aa) / (3 tau_p C_a),  mu_ab = mu_ba = -(P0_ab - P_ab) / (3 tau_p C_ab),
  h_k = mu_k h_{k-1}.
For npt_scr the residual mu - drift is the component noise, whose variance
must match 2 c kT / V (diagonal) and c kT / V (shear) with c = 1 / (3 tau_p C)
in inverse natural pressure units.
"""
import numpy as np
import pytest

import workloads
from conftest import potential

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

KB = 8.617343e-5          # eV/K
P_UNIT = 1.602177e2       # GPa per eV/A^3
COLS = {"sxx": 3, "syy": 4, "szz": 5, "syz": 6, "sxz": 7, "sxy": 8}
COMP = [("sxx", 0, 0), ("syy", 1, 1), ("szz", 2, 2), ("syz", 1, 2), ("sxz", 0, 2),
        ("sxy", 0, 1)]


def _box(row):
    a, b, c = row[9:12], row[12:15], row[15:18]
    return np.array([a, b, c]).T          # columns are the cell vectors


def _mu(row, p0, mod, tau, nc):
    mu = np.eye(3)
    for k in range(nc):
        name, r, c = COMP[k]
        m = -(p0[k] - row[COLS[name]]) / (3.0 * tau * mod[k])
        mu[r, c] += m
        if r != c:
            mu[c, r] += m
    return mu


def _md(kind, h, seed=5):
    import nepx
    t, _, p = workloads.diamond(a=3.567, ncell=5, jitter=0.05, seed=seed)
    frac = np.linalg.solve(np.diag([3.567 * 5] * 3), p)
    pos = np.asarray(h).reshape(3, 3) @ frac
    masses = np.full(len(t), 12.011)
    v = workloads.maxwell_boltzmann(masses, 300.0, seed=seed + 1)
    pot = nepx.Potential(potential("nep_C.txt"), max_atoms=len(t))
    md = nepx.MD(pot, t, masses, pos, v, np.asarray(h, dtype=np.float64))
    return pot, md, len(t)


CUBE = [17.835, 0, 0, 0, 17.835, 0, 0, 0, 17.835]
SHEARED = [17.835, 0.9, 0.4, 0, 17.835, 0.7, 0, 0, 17.835]


@pytest.mark.parametrize("coupling,h", [("anisotropic", CUBE), ("triclinic", SHEARED)])
def test_berendsen_component_update(coupling, h):
    pot, md, n = _md("npt_ber", h)
    nc = 3 if coupling == "anisotropic" else 6
    p0 = [1.0, -0.5, 2.0, 0.3, -0.2, 0.1][:nc]
    mod = [400.0, 300.0, 500.0, 200.0, 250.0, 300.0][:nc]
    tau = 200.0
    md.set_ensemble("npt_ber", T0=300.0, Tdamp=100.0, p_gpa=0.0, bulk_gpa=400.0, tau_p=tau)
    md.set_barostat(coupling, p0, mod)
    rows = md.run(60, 1.0, thermo_every=1)
    prev = np.asarray(h, dtype=np.float64).reshape(3, 3)
    for row in rows:
        want = _mu(row, p0, mod, tau, nc) @ prev
        got = _box(row)
        assert np.allclose(got, want, rtol=1e-12, atol=1e-12), (got, want)
        prev = got
    assert not np.allclose(prev, np.asarray(h).reshape(3, 3))   # the box did move
    if coupling == "anisotropic":
        off = prev - np.diag(np.diag(prev))
        assert np.all(off == 0.0)
    md.close()
    pot.close()


def test_scr_component_noise_amplitude():
    pot, md, n = _md("npt_scr", SHEARED, seed=9)
    p0 = [0.0] * 6
    mod = [400.0] * 6
    tau = 100.0
    md.set_ensemble("npt_scr", T0=300.0, Tdamp=100.0, p_gpa=0.0, bulk_gpa=400.0, tau_p=tau)
    md.set_barostat("triclinic", p0, mod)
    rows = md.run(400, 1.0, thermo_every=1)
    prev = np.asarray(SHEARED, dtype=np.float64).reshape(3, 3)
    eta = [[] for _ in range(6)]
    for row in rows:
        got = _box(row)
        mu = got @ np.linalg.inv(prev)
        drift = _mu(row, p0, mod, tau, 6)
        V = abs(np.linalg.det(prev))
        c = P_UNIT / (3.0 * tau * 400.0)
        for k, (_, r, q) in enumerate(COMP):
            amp = np.sqrt((2.0 if r == q else 1.0) * c * KB * 300.0 / V)
            eta[k].append((mu[r, q] - drift[r, q]) / amp)
        prev = got
    for k in range(6):
        e = np.array(eta[k])
        assert abs(e.mean()) < 0.25 and 0.7 < e.var() < 1.4, (k, e.mean(), e.var())
    md.close()
    pot.close()


def test_isotropic_coupling_rejects_triclinic_box():
    import nepx
    pot, md, n = _md("npt_ber", SHEARED)
    md.set_ensemble("npt_ber", T0=300.0, Tdamp=100.0, p_gpa=0.0, bulk_gpa=400.0, tau_p=200.0)
    with pytest.raises(nepx.NepxError, match="orthogonal"):
        md.run(5, 1.0)
    md.close()
    pot.close()


def test_isotropic_berendsen_against_the_reference_formulas():
    """The reference's isotropic npt_ber (ensemble_control.cpp:180-306,
    box_control.cpp:9-68), restated from the thermo rows: each step's box
    factor is 1 - (P0 - P)/(3 tau_p B) with P the mean of the three normal
    stresses, the box scales by it, and the Berendsen velocity factor is
    sqrt(1 + (T0 / T - 1) / Tdamp) with T the step's temperature."""
    pot, md, n = _md("npt_ber", CUBE)
    tau, bulk, p0, t0, tdamp = 150.0, 300.0, 0.5, 300.0, 80.0
    md.set_ensemble("npt_ber", T0=t0, Tdamp=tdamp, p_gpa=p0, bulk_gpa=bulk, tau_p=tau)
    rows = md.run(50, 1.0, thermo_every=1)
    prev = np.asarray(CUBE, dtype=np.float64).reshape(3, 3)
    for row in rows:
        p_inst = (row[COLS["sxx"]] + row[COLS["syy"]] + row[COLS["szz"]]) / 3.0
        bf = 1.0 - (p0 - p_inst) / (3.0 * tau * bulk)
        assert row[19] == pytest.approx(bf, rel=1e-13, abs=1e-15)
        got = _box(row)
        assert np.allclose(got, bf * prev, rtol=1e-13, atol=1e-13)
        vf = np.sqrt(1.0 + (t0 / row[0] - 1.0) / tdamp)
        assert row[18] == pytest.approx(vf, rel=1e-12)
        prev = got
    md.close()
    pot.close()
