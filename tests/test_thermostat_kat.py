"""Known-answer tests of the stochastic thermostat stream.

The reference pins GPUMD's SVR functions bit for bit
(tests/thermostats/fixtures/svr.json: Gaussian draws, sums of squared
noises and kinetic-energy resamplings per seed / ndeg / tau).  The engine's
host stream (dmg-md_b200/csrc/svr_rng.h) must reproduce every value exactly.
"""
import ctypes
import json
import os
import struct
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    out = tmp_path_factory.mktemp("svr") / "libsvr_harness.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off",
                    os.path.join(ROOT, "tests", "cpp", "svr_harness.cpp"), "-o", str(out)],
                   check=True)
    lib = ctypes.CDLL(str(out))
    dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
    ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
    lib.svr_fixture.argtypes = [ctypes.c_uint32, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                ctypes.c_double, ip, ctypes.c_int, ctypes.c_int, dp, dp, dp]
    lib.svr_step_draws.argtypes = [ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]
    lib.resample.restype = ctypes.c_double
    lib.resample.argtypes = [ctypes.c_double] * 2 + [ctypes.c_int] + [ctypes.c_double] * 3
    return lib


def bits(x):
    return struct.unpack("<Q", struct.pack("<d", float(x)))[0]


def test_svr_fixture_bit_exact(harness):
    fx = json.load(open(os.path.join(GOLDEN, "thermostats", "svr.json")))
    assert len(fx["cases"]) == 16
    for c in fx["cases"]:
        nn = np.array(c["sumnoises_nn"], dtype=np.int32)
        g = np.zeros(6)
        s = np.zeros(len(nn))
        r = np.zeros(c["resamplekin_steps"])
        harness.svr_fixture(c["seed"], c["ndeg"], c["taut"], c["kk"], c["sigma"], nn, len(nn),
                            len(r), g, s, r)
        assert [bits(v) for v in g] == c["gasdev_bits"], c["seed"]
        assert [bits(v) for v in s] == [e["bits"] for e in c["sumnoises"]]
        assert [bits(v) for v in r] == c["resamplekin_bits"], (c["seed"], c["ndeg"], c["taut"])


def test_nhc_fixture_bit_exact(harness):
    """Nose-Hoover chain states and factors of tests/thermostats/fixtures/nhc.json."""
    fx = json.load(open(os.path.join(GOLDEN, "thermostats", "nhc.json")))
    dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
    harness.nhc_step.restype = ctypes.c_double
    harness.nhc_step.argtypes = [dp, dp, dp] + [ctypes.c_double] * 4

    def unhex(h):
        return struct.unpack("<d", struct.pack("<Q", int(h, 16)))[0]

    for c in fx["cases"]:
        pos = np.array([unhex(x) for x in c["initial_position"]])
        mom = np.array([unhex(x) for x in c["initial_momentum"]])
        mass = np.array([unhex(x) for x in c["initial_mass"]])
        ek2 = c["initial_Ek2"]
        for s in c["steps"]:
            f = harness.nhc_step(pos, mom, mass, ek2, 8.617343e-5 * s["target_temperature"],
                                 3.0 * c["N"], 0.5 * c["dt"])
            ek2 *= f * f
            assert bits(f) == int(s["factor"], 16), c["name"]
            assert bits(ek2) == int(s["Ek2_after"], 16)
            assert [bits(v) for v in pos] == [int(x, 16) for x in s["position"]]
            assert [bits(v) for v in mom] == [int(x, 16) for x in s["momentum"]]
