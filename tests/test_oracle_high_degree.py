"""The CPU oracle at l_max 5..8 (the reference GPU path's harmonics go to
degree 8: NUM_OF_ABC = 80, src/gpumd_compat/nep_utilities.cuh:50).

The harmonic tables come from Rodrigues' formula; the tests check them
against the Legendre recurrences and closed forms, and the whole evaluation
through properties every correct NEP has: energy invariant under rotation,
forces equal to -dE/dr, virial trace equal to -dE/d(ln volume).
"""
import math

import numpy as np
import pytest

import oracle
import workloads


def test_tables_are_legendre_derivatives():
    z_tab, c3b = oracle.harmonic_tables()
    z = np.linspace(-0.9, 0.9, 13)
    for L in range(1, 9):
        for m in range(0, L + 1):
            # numerical m-th derivative of P_L through its polynomial fit
            coeff = np.polynomial.legendre.leg2poly([0] * L + [1])
            for _ in range(m):
                coeff = np.polynomial.polynomial.polyder(coeff)
            exact = np.polynomial.polynomial.polyval(z, coeff)
            ours = np.polynomial.polynomial.polyval(z, z_tab[L, m, :L - m + 1])
            kappa = exact[np.argmax(np.abs(ours))] / ours[np.argmax(np.abs(ours))]
            assert np.allclose(exact, kappa * ours, rtol=1e-12, atol=1e-12)
            # primitive integer polynomial with a positive leading coefficient
            ints = z_tab[L, m, :L - m + 1]
            assert np.all(ints == np.round(ints)) and ints[L - m] > 0
            assert np.gcd.reduce(np.abs(ints).astype(np.int64)) == 1
            w = (2 * L + 1) / (4 * math.pi) * math.factorial(L - m) / math.factorial(L + m)
            st = L * L - 1
            idx = [st] if m == 0 else [st + 2 * m - 1, st + 2 * m]
            for k in idx:
                assert c3b[k] == pytest.approx(w * kappa * kappa, rel=1e-12)


def test_q_l_is_addition_theorem():
    """sum_m weight * Y^2 at one direction equals (2L+1)/(4 pi): the
    addition theorem, which fixes the weight of every degree."""
    z_tab, c3b = oracle.harmonic_tables()
    rng = np.random.default_rng(0)
    for _ in range(5):
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        for L in range(1, 9):
            st = L * L - 1
            total = 0.0
            for m in range(L + 1):
                zf = np.polynomial.polynomial.polyval(u[2], z_tab[L, m, :L - m + 1])
                c = complex(u[0], u[1]) ** m
                if m == 0:
                    total += c3b[st] * zf * zf
                else:
                    total += 2 * c3b[st + 2 * m - 1] * zf * zf * (c.real ** 2 + c.imag ** 2)
            assert total == pytest.approx((2 * L + 1) / (4 * math.pi), rel=1e-12)


def _rotation(seed):
    q, _ = np.linalg.qr(np.random.default_rng(seed).normal(size=(3, 3)))
    return q if np.linalg.det(q) > 0 else -q


@pytest.mark.parametrize("l_max", [(6, 2, 1), (8, 0, 0), (8, 2, 1)])
def test_high_degree_invariance_and_forces(tmp_path, l_max):
    path = workloads.write_nep(str(tmp_path / "nep.txt"), symbols=("C", "H"), rc=(4.5, 4.0),
                               n_max=(3, 3), basis=(6, 6), l_max=l_max, H=12, seed=5)
    m = oracle.OracleModel(path)
    rng = np.random.default_rng(2)
    n = 24
    pos = rng.uniform(-3.5, 3.5, (3, n))
    keep = np.ones(n, bool)
    for i in range(n):   # keep atoms at least 1.1 A apart
        d = np.linalg.norm(pos[:, :i][:, keep[:i]] - pos[:, i:i + 1], axis=0)
        keep[i] = d.size == 0 or d.min() > 1.1
    pos = pos[:, keep]
    n = pos.shape[1]
    types = rng.integers(0, 2, n)
    h = [40.0, 0, 0, 0, 40.0, 0, 0, 0, 40.0]
    pbc = [0, 0, 0]
    pe, f, w = m.compute(types, h, pos + 20.0, pbc)
    assert np.isfinite(pe).all() and abs(pe.sum()) > 0
    R = _rotation(7)
    pe_r, f_r, _ = m.compute(types, h, R @ pos + 20.0, pbc)
    assert np.allclose(pe_r, pe, rtol=1e-10, atol=1e-12)
    assert np.allclose(f_r, R @ f, rtol=1e-8, atol=1e-10)
    eps = 1e-5
    for i in (0, n // 2):
        for d in range(3):
            p1, p2 = pos.copy(), pos.copy()
            p1[d, i] += eps
            p2[d, i] -= eps
            e1 = m.compute(types, h, p1 + 20.0, pbc)[0].sum()
            e2 = m.compute(types, h, p2 + 20.0, pbc)[0].sum()
            assert abs(-(e1 - e2) / (2 * eps) - f[d, i]) < 1e-6 * max(1.0, abs(f[d, i]))
    assert abs(f.sum(axis=1)).max() < 1e-9
