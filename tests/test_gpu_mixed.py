"""The mixed-precision path: the ANN on the tensor cores (tcgen05 MMAs inside
the descriptor kernel, 16-bit operands, FP32 accumulation in TMEM).

Descriptors and forces stay FP32; only the two ANN contractions take 16-bit
operands: FP16 with per-layer power-of-two scaling ("mixed", 11 significant
bits) or BF16 ("mixed_bf16", 8).  Tolerances against the FP64 oracle, per
format (REL): relative 2-norm of the force errors, per-atom energy errors
of REL times the largest |site energy| plus 1e-5 eV, and relative 2-norm of
the per-atom virial errors of 2.5 REL (the virial sums r (x) f over edges
whose contributions partly cancel).
Against the plain FP32 path the same relative bound holds.  Tiles that hold
several center types (multi-type systems), the explicit-row path and MD run
through the same kernel.
"""
import numpy as np
import pytest

import oracle
import workloads
from conftest import potential

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

REL = {"mixed": 2e-3, "mixed_bf16": 1.6e-2}
FORMATS = sorted(REL)


def _both(path, t, h, p, prec, pbc=(1, 1, 1)):
    import nepx
    pot = nepx.Potential(path, max_atoms=len(t))
    tt = torch.as_tensor(np.asarray(t, dtype=np.int32), device="cuda")
    pp = torch.as_tensor(np.ascontiguousarray(p), device="cuda")
    r32 = [x.cpu().numpy() for x in pot.compute(tt, h, pp, pbc=pbc, sync_check=True)]
    pot.set_precision(prec)
    rmx = [x.cpu().numpy() for x in pot.compute(tt, h, pp, pbc=pbc, sync_check=True)]
    return r32, rmx


def assert_mixed_close(ref, got, label, prec):
    """Mixed-precision results (pe, f, w) against FP64 ones at REL[prec]."""
    pe0, f0, w0 = ref
    rel = REL[prec]
    ef = np.linalg.norm(got[1] - f0) / np.linalg.norm(f0)
    assert ef <= rel, "%s %s force rel err vs FP64 %g" % (label, prec, ef)
    de = np.abs(got[0] - pe0).max()
    scale = np.abs(pe0).max()
    assert de <= 1e-5 + rel * scale, "%s %s max dE %g (|E| %g)" % (label, prec, de, scale)
    ew = np.linalg.norm(got[2] - w0) / np.linalg.norm(w0)
    assert ew <= 2.5 * rel, "%s %s virial rel err %g" % (label, prec, ew)


def _check(ref, r32, rmx, label, prec):
    assert_mixed_close(ref, rmx, label, prec)
    e32 = np.linalg.norm(rmx[1] - r32[1]) / np.linalg.norm(r32[1])
    assert e32 <= REL[prec], "%s %s vs fp32 %g" % (label, prec, e32)


@pytest.mark.parametrize("prec", FORMATS)
def test_mixed_small_water(prec):
    t, h, p = workloads.water(n_mol=100, seed=2)     # 300 atoms: 10 CTAs, two types each
    path = potential("nep_water.txt")
    r32, rmx = _both(path, t, h, p, prec)
    _check(oracle.OracleModel(path).compute(t, h, p), r32, rmx, "water 300", prec)


@pytest.mark.parametrize("prec", FORMATS)
def test_mixed_water_and_carbon(prec):
    for name, (t, h, p) in (("nep_water.txt", workloads.water(n_mol=700, seed=1)),
                            ("nep_C.txt", workloads.diamond(ncell=6, jitter=0.08, seed=2))):
        path = potential(name)
        r32, rmx = _both(path, t, h, p, prec)
        _check(oracle.OracleModel(path).compute(t, h, p), r32, rmx, name, prec)


@pytest.mark.parametrize("prec", FORMATS)
def test_mixed_multitype_nep5(tmp_path, prec):
    path = workloads.write_nep(str(tmp_path / "nep.txt"), version=5, symbols=("C", "H", "O", "Cu"),
                               zbl=(1.0, 2.0), rc=(5.0, 4.0), mn=(160, 80), H=64, seed=17,
                               std=0.1, q_scaler=0.05)
    t, h, p = workloads.random_packed(n=1500, num_types=4, density=0.08, seed=9)
    r32, rmx = _both(path, t, h, p, prec)
    _check(oracle.OracleModel(path).compute(t, h, p), r32, rmx, "nep5 4 types", prec)


def test_mixed_large_hidden_layer(tmp_path):
    """200 hidden units: GEMM1 in two passes of 128 rows, GEMM2 over K = 208."""
    path = workloads.write_nep(str(tmp_path / "nep.txt"), version=4, symbols=("O", "H"),
                               rc=(6.0, 4.0), mn=(250, 100), n_max=(8, 8), l_max=(4, 2, 1),
                               H=200, seed=23, std=0.1, q_scaler=0.02)
    t, h, p = workloads.water(n_mol=500, seed=3)
    r32, rmx = _both(path, t, h, p, "mixed")
    _check(oracle.OracleModel(path).compute(t, h, p), r32, rmx, "H 200", "mixed")


def test_mixed_small_box_and_md():
    import nepx
    t, h, p = workloads.diamond(ncell=2, jitter=0.03, seed=41)     # small box
    path = potential("nep_C.txt")
    r32, rmx = _both(path, t, h, p, "mixed")
    _check(oracle.OracleModel(path).compute(t, h, p), r32, rmx, "small box", "mixed")
    t, h, p = workloads.diamond(ncell=5, jitter=0.03, seed=42)
    masses = np.full(len(t), 12.011)
    v = workloads.maxwell_boltzmann(masses, 300.0, seed=43)
    pot = nepx.Potential(path, max_atoms=len(t))
    pot.set_precision("mixed")
    md = nepx.MD(pot, t, masses, p, v, h)
    md.set_ensemble("nve")
    rows = md.run(600, 0.5, thermo_every=20)
    etot = (rows[:, 1] + rows[:, 2]) / len(t)
    assert np.abs(etot - etot.mean()).max() < 2e-4
