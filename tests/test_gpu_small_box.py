"""GPU parity of the small-box (explicit-row) path.

A box thinner than 2.5 (rc + 1) in a periodic direction takes the reference's
small-box path (nep.cu:2002-2100, nep_small_box.cuh): neighbours over every
atom and every image of the expanded box, rows rebuilt at every call.  The
engine's explicit-row kernels must give

  * the reference suite's golden values for single_small_static (8 C atoms);
  * the FP64 oracle's values at the tolerances of test_gpu_force.py;
  * the reference's own FP32 GPU small-box path within 1e-5 relative force
    and 1e-6 eV/atom, with identical neighbour rows (same image order);
  * an NVE trajectory that conserves energy.
"""
import os

import numpy as np
import pytest

import oracle
import workloads
from conftest import potential
from test_gpu_force import ROWMAJOR, assert_close, run_gpu

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_golden_small_static(goldens):
    rec = goldens["static"]["single_small_static"]
    path = potential(rec["potential"])
    pos = np.array(rec["pos"]).T
    ref = oracle.OracleModel(path).compute(rec["type"], rec["h"], pos, rec["pbc"])
    _, pe, f, w = run_gpu(path, rec["type"], rec["h"], pos, rec["pbc"])
    assert_close(ref, (pe, f, w), "single_small_static")
    fg = np.array(rec["force"]).T
    assert np.all(np.abs(f - fg) <= 1e-6 + 1e-4 * np.abs(fg))
    eg = np.array(rec["energy_atom"])
    assert np.all(np.abs(pe - eg) <= 1e-8 + 1e-5 * np.abs(eg) + 2e-5)
    wg = np.array(rec["virial_rowmajor"]).T
    assert np.all(np.abs(w[ROWMAJOR] - wg) <= 1e-6 + 1e-4 * np.abs(wg) + 2e-5)


def _thin_triclinic(n, seed):
    rng = np.random.default_rng(seed)
    H = np.array([[7.5, 1.1, 0.6], [0.0, 21.0, 1.4], [0.0, 0.0, 19.0]])
    frac = rng.uniform(0, 1, (3, n))
    return rng.integers(0, 2, n).astype(np.int32), H.reshape(-1), H @ frac


@pytest.mark.parametrize("case", ["water_cube", "thin_triclinic", "slab_pbc_xy"])
def test_small_box_matches_oracle(case):
    path = potential("nep_water.txt")
    pbc = (1, 1, 1)
    if case == "water_cube":
        t, h, p = workloads.water(n_mol=30, seed=3)       # L ~ 9.7 A
    elif case == "thin_triclinic":
        t, h, p = _thin_triclinic(250, 4)
    else:
        t, h, p = workloads.water(n_mol=40, seed=5)
        h = np.array(h, dtype=np.float64).reshape(3, 3) * np.diag([1.0, 1.0, 3.0])
        h = h.reshape(-1)
        pbc = (1, 1, 0)
    ref = oracle.OracleModel(path).compute(t, h, p, pbc)
    _, pe, f, w = run_gpu(path, t, h, p, pbc)
    assert_close(ref, (pe, f, w), case)


def test_small_box_multitype_zbl(tmp_path):
    syms = ("C", "H", "O", "Cu")
    path = workloads.write_nep(str(tmp_path / "nep.txt"), version=5, symbols=syms,
                               zbl=(1.0, 2.0), rc=(5.0, 4.0), mn=(200, 100), H=24, seed=13,
                               std=0.1)
    t, h, p = workloads.random_packed(n=60, num_types=4, density=0.08, seed=6)
    ref = oracle.OracleModel(path).compute(t, h, p)
    _, pe, f, w = run_gpu(path, t, h, p)
    assert_close(ref, (pe, f, w), "multitype small box")


def test_unsupported_thin_and_thick_box():
    nepx = __import__("nepx")
    t, _, p = workloads.water(n_mol=30, seed=3)
    h = np.diag([9.7, 9.7, 80.0]).reshape(-1)   # thin in x, y; z > 10 rc
    pot = nepx.Potential(potential("nep_water.txt"), max_atoms=len(t))
    with pytest.raises(nepx.NepxError) as err:
        pot.compute(torch.as_tensor(t, device="cuda"), h, torch.as_tensor(p, device="cuda"))
    assert err.value.code == 8


def _small_vs_reference(path, t, h, p, tmp_path):
    import nepx
    n = len(t)
    cwd = os.getcwd()
    os.chdir(tmp_path)   # the reference appends neighbor.out to the working directory
    try:
        tt = torch.as_tensor(np.asarray(t, dtype=np.int32), device="cuda")
        pp = torch.as_tensor(np.ascontiguousarray(p), device="cuda")
        ref = oracle.RefGpuModel(path, n)
        ref.set_atoms(tt, pp)
        out_r = [torch.empty(n, dtype=torch.float64, device="cuda"),
                 torch.empty(3, n, dtype=torch.float64, device="cuda"),
                 torch.empty(9, n, dtype=torch.float64, device="cuda")]
        ref.compute(h, out=out_r)
        pot = nepx.Potential(path, max_atoms=n)
        out_m = pot.compute(tt, h, pp, sync_check=True)
        torch.cuda.synchronize()
        pe0, f0, w0 = [x.cpu().numpy() for x in out_r]
        pe1, f1, w1 = [x.cpu().numpy() for x in out_m]
        assert np.linalg.norm(f1 - f0) / np.linalg.norm(f0) <= 1e-5
        assert abs(pe1.sum() - pe0.sum()) / n <= 1e-6
        assert np.linalg.norm(w1 - w0) / np.linalg.norm(w0) <= 2e-5
        for which, mn in ((0, pot.info["MN_r"]), (1, pot.info["MN_a"])):
            a = ref.neighbors(which, mn, small=True)
            b = pot.neighbors(which, n)
            for i in range(n):
                assert np.array_equal(a[i], b[i]), (which, i)
    finally:
        os.chdir(cwd)


@pytest.mark.skipif(not oracle.ref_gpu_available(), reason="reference GPU library not built")
def test_small_box_matches_reference_gpu(tmp_path):
    t, h, p = workloads.water(n_mol=40, seed=11)          # L ~ 10.6 A
    _small_vs_reference(potential("nep_water.txt"), t, h, p, tmp_path)


@pytest.mark.skipif(not oracle.ref_gpu_available(), reason="reference GPU library not built")
@pytest.mark.parametrize("case", ["zbl_universal", "zbl_flexible", "typewise_cutoffs"])
def test_small_box_models_match_reference_gpu(tmp_path, case):
    """The small-box path of the reference (its image rows and its small-box
    ZBL) for four-type NEP5 with universal or flexible ZBL, and for per-type
    cutoffs."""
    syms = ("C", "H", "O", "Cu")
    zbl = {"zbl_universal": (1.0, 2.0), "zbl_flexible": "flexible",
           "typewise_cutoffs": None}[case]
    rc = ((5.0, 4.0), (4.2, 3.6), (4.6, 3.8), (5.0, 4.0)) if case == "typewise_cutoffs" \
        else (5.0, 4.0)
    path = workloads.write_nep(str(tmp_path / "nep.txt"), version=5, symbols=syms, zbl=zbl,
                               rc=rc, mn=(200, 100), H=24, seed=47, q_scaler=0.1)
    t, h, p = workloads.random_packed(n=60, num_types=4, density=0.08, seed=53)
    _small_vs_reference(path, t, h, p, tmp_path)


def test_small_box_nve_conserves_energy():
    nepx = __import__("nepx")
    t, h, p = workloads.diamond(ncell=2, jitter=0.03, seed=21)   # 64 atoms, L = 7.1 A
    masses = np.full(len(t), 12.011)
    v = workloads.maxwell_boltzmann(masses, 300.0, seed=22)
    pot = nepx.Potential(potential("nep_C.txt"), max_atoms=len(t))
    md = nepx.MD(pot, t, masses, p, v, h)
    md.set_ensemble("nve")
    rows = md.run(400, 0.5, thermo_every=10)
    etot = (rows[:, 1] + rows[:, 2]) / len(t)
    assert np.abs(etot - etot.mean()).max() < 5e-4
    s = md.state()
    ref = oracle.OracleModel(potential("nep_C.txt")).compute(t, s["h"], s["pos"])
    assert np.linalg.norm(s["force"] - ref[1]) / np.linalg.norm(ref[1]) < 2e-5
