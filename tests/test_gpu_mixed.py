"""The mixed-precision path: the ANN on the tensor cores (tcgen05, 3xTF32).

Descriptors and forces stay FP32; only the two ANN contractions move to the
tensor cores.  Against the FP64 oracle the forces must keep an RMSE of at
most 1e-4 eV/A and per-atom energies 2e-5 eV; against the plain FP32 path the
relative force difference stays at FP32 rounding (1e-5).  Tiles that hold
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


def _both(path, t, h, p, pbc=(1, 1, 1)):
    import nepx
    pot = nepx.Potential(path, max_atoms=len(t))
    tt = torch.as_tensor(np.asarray(t, dtype=np.int32), device="cuda")
    pp = torch.as_tensor(np.ascontiguousarray(p), device="cuda")
    r32 = [x.cpu().numpy() for x in pot.compute(tt, h, pp, pbc=pbc, sync_check=True)]
    pot.set_precision("mixed")
    rmx = [x.cpu().numpy() for x in pot.compute(tt, h, pp, pbc=pbc, sync_check=True)]
    return r32, rmx


def _check(ref, r32, rmx, label):
    pe0, f0, w0 = ref
    rmse = np.sqrt(np.mean((rmx[1] - f0) ** 2))
    assert rmse <= 1e-4, "%s force RMSE vs FP64 %g" % (label, rmse)
    assert np.abs(rmx[0] - pe0).max() <= 2e-5 + 2e-6 * np.abs(pe0).max(), label
    rel = np.linalg.norm(rmx[1] - r32[1]) / np.linalg.norm(r32[1])
    assert rel <= 1e-5, "%s mixed vs fp32 %g" % (label, rel)
    assert np.linalg.norm(rmx[2] - w0) / np.linalg.norm(w0) <= 5e-5, label


def test_mixed_small_water():
    t, h, p = workloads.water(n_mol=100, seed=2)     # 300 atoms: three tiles, two types
    path = potential("nep_water.txt")
    r32, rmx = _both(path, t, h, p)
    _check(oracle.OracleModel(path).compute(t, h, p), r32, rmx, "water 300")


def test_mixed_water_and_carbon():
    for name, (t, h, p) in (("nep_water.txt", workloads.water(n_mol=700, seed=1)),
                            ("nep_C.txt", workloads.diamond(ncell=6, jitter=0.08, seed=2))):
        path = potential(name)
        r32, rmx = _both(path, t, h, p)
        _check(oracle.OracleModel(path).compute(t, h, p), r32, rmx, name)


def test_mixed_multitype_nep5(tmp_path):
    path = workloads.write_nep(str(tmp_path / "nep.txt"), version=5, symbols=("C", "H", "O", "Cu"),
                               zbl=(1.0, 2.0), rc=(5.0, 4.0), mn=(160, 80), H=64, seed=17,
                               std=0.1, q_scaler=0.05)
    t, h, p = workloads.random_packed(n=1500, num_types=4, density=0.08, seed=9)
    r32, rmx = _both(path, t, h, p)
    _check(oracle.OracleModel(path).compute(t, h, p), r32, rmx, "nep5 4 types")


def test_mixed_small_box_and_md():
    import nepx
    t, h, p = workloads.diamond(ncell=2, jitter=0.03, seed=41)     # small box
    path = potential("nep_C.txt")
    r32, rmx = _both(path, t, h, p)
    _check(oracle.OracleModel(path).compute(t, h, p), r32, rmx, "small box")
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
