"""GPU parity at l_max 5..8.

The reference GPU path evaluates harmonics up to degree 8 (NUM_OF_ABC = 80,
src/gpumd_compat/nep_utilities.cuh:50; Z_COEFFICIENT_5..8 at :137-187).  The
engine runs such models through its LMAX-8 kernel instances (80 moment
components per radial function).  Checked here against the FP64 oracle on
the large-box, small-box, batched and mixed-precision paths, and against the
reference's own FP32 GPU kernels.
"""
import os

import numpy as np
import pytest

import oracle
import workloads
from test_gpu_force import assert_close, run_gpu
from test_gpu_mixed import assert_mixed_close

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

L_MAX = [(6, 2, 1), (8, 0, 0), (8, 2, 1)]


def _model(tmp_path, l_max, version=4):
    return workloads.write_nep(str(tmp_path / ("nep_l%d_%d%d.txt" % l_max)), version=version,
                               symbols=("O", "H"), rc=(5.0, 4.0), mn=(150, 80), n_max=(4, 4),
                               basis=(8, 8), l_max=l_max, H=20, seed=11, q_scaler=0.1)


@pytest.mark.parametrize("l_max", L_MAX)
def test_large_box_matches_oracle(tmp_path, l_max):
    path = _model(tmp_path, l_max)
    t, h, p = workloads.water(n_mol=200, seed=21)       # 600 atoms, ~18 A cube
    ref = oracle.OracleModel(path).compute(t, h, p)
    _, pe, f, w = run_gpu(path, t, h, p)
    assert_close(ref, (pe, f, w), "l_max %s large box" % (l_max,))


@pytest.mark.parametrize("l_max", [(8, 2, 1)])
def test_small_box_and_nep5_match_oracle(tmp_path, l_max):
    path = _model(tmp_path, l_max, version=5)
    t, h, p = workloads.water(n_mol=30, seed=22)        # ~9.7 A cube: small-box path
    ref = oracle.OracleModel(path).compute(t, h, p)
    _, pe, f, w = run_gpu(path, t, h, p)
    assert_close(ref, (pe, f, w), "l_max 8 small box")


def test_batch_and_mixed_precision(tmp_path):
    import nepx
    path = _model(tmp_path, (8, 2, 1))
    structs = [workloads.water(n_mol=30, seed=23), workloads.water(n_mol=250, seed=24),
               workloads.water(n_mol=45, seed=25)]
    total = sum(len(s[0]) for s in structs)
    pot = nepx.Potential(path, max_atoms=total)
    tt = torch.as_tensor(np.concatenate([np.asarray(s[0], np.int32) for s in structs]),
                         device="cuda")
    pp = torch.as_tensor(np.ascontiguousarray(np.concatenate([s[2] for s in structs], axis=1)),
                         device="cuda")
    descs = [(len(s[0]), s[1], (1, 1, 1)) for s in structs]
    orc = oracle.OracleModel(path)
    for precision in ("fp32", "mixed"):
        pot.set_precision(precision)
        pe, f, w = [x.cpu().numpy() for x in pot.compute_batch(descs, tt, pp, sync_check=True)]
        o = 0
        for k, (t, h, p) in enumerate(structs):
            n = len(t)
            got = (pe[o:o + n], f[:, o:o + n], w[:, o:o + n])
            label = "%s struct %d" % (precision, k)
            if precision == "fp32":
                assert_close(orc.compute(t, h, p), got, label)
            else:
                assert_mixed_close(orc.compute(t, h, p), got, label, precision)
            o += n


def test_nve_energy_conserved(tmp_path):
    import nepx
    path = _model(tmp_path, (8, 2, 1))
    t, h, p = workloads.water(n_mol=200, seed=26)
    masses = np.where(np.asarray(t) == 0, 15.999, 1.008)
    v = workloads.maxwell_boltzmann(masses, 300.0, seed=27)
    pot = nepx.Potential(path, max_atoms=len(t))
    md = nepx.MD(pot, t, masses, p, v, h)
    md.set_ensemble("nve")
    rows = md.run(400, 0.25, thermo_every=20)
    e = (rows[:, 1] + rows[:, 2]) / len(t)
    assert np.isfinite(e).all()
    assert np.abs(e - e[0]).max() < 2e-4, np.abs(e - e[0]).max()
    md.close()
    pot.close()


@pytest.mark.skipif(not oracle.ref_gpu_available(), reason="reference GPU library not built")
@pytest.mark.parametrize("l_max", [(6, 2, 1), (8, 2, 1)])
def test_matches_reference_gpu(tmp_path, l_max):
    import nepx
    path = _model(tmp_path, l_max)
    t, h, p = workloads.water(n_mol=500, seed=28)
    n = len(t)
    tt = torch.as_tensor(np.asarray(t, dtype=np.int32), device="cuda")
    pp = torch.as_tensor(np.ascontiguousarray(p), device="cuda")
    cwd = os.getcwd()
    os.chdir(tmp_path)   # the reference appends neighbor.out to the working directory
    try:
        ref = oracle.RefGpuModel(path, n)
        ref.set_atoms(tt, pp)
        out_r = [torch.empty(n, dtype=torch.float64, device="cuda"),
                 torch.empty(3, n, dtype=torch.float64, device="cuda"),
                 torch.empty(9, n, dtype=torch.float64, device="cuda")]
        ref.compute(h, out=out_r)
        torch.cuda.synchronize()
    finally:
        os.chdir(cwd)
    pe0, f0, w0 = [x.cpu().numpy() for x in out_r]
    pot = nepx.Potential(path, max_atoms=n)
    pe1, f1, w1 = [x.cpu().numpy() for x in pot.compute(tt, h, pp, sync_check=True)]
    rel_f = np.linalg.norm(f1 - f0) / np.linalg.norm(f0)
    assert rel_f <= 1e-5, rel_f
    assert abs(pe1.sum() - pe0.sum()) / n <= 1e-6
    assert np.linalg.norm(w1 - w0) / np.linalg.norm(w0) <= 2e-5
