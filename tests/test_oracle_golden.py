"""Pins the FP64 CPU oracle against the reference's golden vectors.

The goldens are GPUMD 5.9.1 FP32 outputs of DMG-MD's tests/baseline suite
(small-box and large-box carbon, two-type water, three-type NEP-ZBL).  The
reference suite's own tolerances are force rtol 1e-4 / atol 1e-6 eV/A,
energy rtol 1e-5 / atol 1e-8 eV (tests/baseline/manifest.json:20-35); an FP64
evaluation differs from the FP32 goldens by FP32 rounding, so the oracle is
held to |dF| <= 1e-5 + 1e-6|F|, |dE| <= 2e-5 + 1e-6|E| eV/atom, |dW| <= 1e-5 + 1e-6|W|.
"""
import numpy as np
import pytest

import oracle
from conftest import potential

CASES = ["single_small_static", "single_large_nve", "multi_nvt_restart", "nep_zbl_boundary"]
ROWMAJOR = [0, 3, 4, 6, 1, 5, 7, 8, 2]  # xx yy zz xy xz yz yx zx zy -> row-major


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_gpumd_goldens(goldens, case):
    rec = goldens["static"][case]
    m = oracle.OracleModel(potential(rec["potential"]))
    pe, f, w = m.compute(rec["type"], rec["h"], np.array(rec["pos"]).T, rec["pbc"])
    fg = np.array(rec["force"]).T
    eg = np.array(rec["energy_atom"])
    wg = np.array(rec["virial_rowmajor"]).T
    assert np.all(np.abs(f - fg) <= 1e-5 + 1e-6 * np.abs(fg))
    assert np.all(np.abs(pe - eg) <= 2e-5 + 1e-6 * np.abs(eg))
    assert np.all(np.abs(w[ROWMAJOR] - wg) <= 1e-5 + 1e-6 * np.abs(wg))
    assert abs(pe.sum() - rec["energy_total"]) <= 1e-4 + 1e-6 * abs(rec["energy_total"])


def test_oracle_energy_force_consistency():
    """Central finite differences of the oracle energy reproduce its forces."""
    rng = np.random.default_rng(3)
    n, L = 40, 9.0
    pos = rng.uniform(0, L, (3, n))
    types = rng.integers(0, 2, n)
    h = [L, 0, 0, 0, L, 0, 0, 0, L]
    m = oracle.OracleModel(potential("nep_water.txt"))
    _, f, _ = m.compute(types, h, pos)
    eps = 1e-5
    for i in (0, 7, 19):
        for d in range(3):
            p1 = pos.copy()
            p1[d, i] += eps
            p2 = pos.copy()
            p2[d, i] -= eps
            e1 = m.compute(types, h, p1)[0].sum()
            e2 = m.compute(types, h, p2)[0].sum()
            assert abs(-(e1 - e2) / (2 * eps) - f[d, i]) < 1e-6 * max(1.0, abs(f[d, i]))


def test_oracle_virial_sum_is_pair_virial():
    """Sum of per-atom virials equals -sum over edges r (x) f (translation invariance)."""
    rng = np.random.default_rng(4)
    n, L = 64, 10.0
    pos = rng.uniform(0, L, (3, n))
    types = np.zeros(n, dtype=int)
    h = [L, 0, 0, 0, L, 0, 0, 0, L]
    m = oracle.OracleModel(potential("nep_C.txt"))
    pe, f, w = m.compute(types, h, pos)
    assert abs(f.sum(axis=1)).max() < 1e-9
    # a uniform strain derivative check of the total virial trace
    eps = 1e-6
    e0 = []
    for s in (1 + eps, 1 - eps):
        hs = [L * s, 0, 0, 0, L * s, 0, 0, 0, L * s]
        e0.append(m.compute(types, hs, pos * s)[0].sum())
    dE = (e0[0] - e0[1]) / (2 * eps)
    assert abs(-dE - w[:3].sum()) < 1e-5 * max(1.0, abs(dE))


def test_oracle_flexible_zbl_forces(tmp_path):
    """Flexible (per-pair fitted) ZBL: the oracle's forces are -dE/dr, with
    close contacts inside every pair's inner and outer ZBL cutoff."""
    import workloads
    path = workloads.write_nep(str(tmp_path / "nep.txt"), version=4, symbols=("C", "O"),
                               zbl="flexible", rc=(4.0, 3.5), mn=(80, 60), H=8, seed=21)
    rng = np.random.default_rng(5)
    n, L = 30, 9.0
    pos = rng.uniform(0, L, (3, n))
    pos[:, 1] = pos[:, 0] + [0.7, 0.2, 0.1]      # pairs at 0.7 A and 1.5 A
    pos[:, 3] = pos[:, 2] + [1.4, 0.4, 0.3]
    types = rng.integers(0, 2, n)
    h = [L, 0, 0, 0, L, 0, 0, 0, L]
    m = oracle.OracleModel(path)
    _, f, _ = m.compute(types, h, pos)
    eps = 1e-6
    for i in (0, 1, 2, 3):
        for d in range(3):
            p1 = pos.copy()
            p1[d, i] += eps
            p2 = pos.copy()
            p2[d, i] -= eps
            e1 = m.compute(types, h, p1)[0].sum()
            e2 = m.compute(types, h, p2)[0].sum()
            assert abs(-(e1 - e2) / (2 * eps) - f[d, i]) < 1e-5 * max(1.0, abs(f[d, i]))

