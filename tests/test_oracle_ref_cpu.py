"""Pins the oracle against the reference's own FP64 CPU evaluator.

oracle/_ref/libnep_ref_cpu.so is NEP3_CPU
(third_party/lammps-matpl-overlay/files/src/nep_cpu.cpp) compiled from the
reference sources by oracle/Makefile.  Both are FP64, so agreement is held to
1e-9 relative.  NEP3_CPU accepts a single global cutoff and the q_222/q_1111
invariants only (nep_cpu.cpp:2085-2146), which all cases below satisfy.
"""
import numpy as np
import pytest

import oracle
from conftest import potential

pytestmark = pytest.mark.skipif(not oracle.ref_cpu_available(),
                                reason="reference NEP3_CPU not built (reference tree absent)")


def _check(pot, types, h, pos, threads=2):
    a = oracle.OracleModel(potential(pot)).compute(types, h, pos)
    b = oracle.RefCpuModel(potential(pot)).compute(types, h, pos, threads=threads)
    for x, y in zip(a, b):
        assert np.all(np.abs(x - y) <= 1e-9 * (1.0 + np.abs(y)))


@pytest.mark.parametrize("case", ["single_small_static", "single_large_nve",
                                  "multi_nvt_restart", "nep_zbl_boundary"])
def test_golden_structures(goldens, case):
    rec = goldens["static"][case]
    _check(rec["potential"], rec["type"], rec["h"], np.array(rec["pos"]).T)


def test_random_water_box():
    rng = np.random.default_rng(0)
    n, L = 300, 14.4
    _check("nep_water.txt", rng.integers(0, 2, n), [L, 0, 0, 0, L, 0, 0, 0, L],
           rng.uniform(0, L, (3, n)), threads=4)


def test_triclinic_carbon():
    rng = np.random.default_rng(1)
    n = 120
    h = np.array([[11.0, 1.5, 0.7], [0.0, 10.5, 1.1], [0.0, 0.0, 10.8]])
    frac = rng.uniform(0, 1, (3, n))
    _check("nep_C.txt", np.zeros(n, dtype=int), h.reshape(-1), h @ frac)
