"""GPU parity of the CUDA NEP force path against the FP64 CPU oracle.

Everything goes through the C ABI (lib/libnepx.so via nepx.py).  Tolerances:

  * force: ||F_gpu - F_oracle||_2 / ||F_oracle||_2 <= 2e-5 (FP32 kernels against
    FP64), and per component |dF| <= 1e-4 (1 + |F|);
  * per-atom energy: |dE| <= 2e-5 eV + 2e-6 |E| (FP32 accumulation of an ANN
    with O(1) weights), total energy per atom <= 2e-6 eV;
  * per-atom virial: relative 2-norm <= 5e-5;
  * neighbour sets: identical to the oracle's FP32 predicate, except pairs
    whose squared distance is within 4 float ulp of the cutoff.
"""
import numpy as np
import pytest

import oracle
import workloads
from conftest import potential

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

ROWMAJOR = [0, 3, 4, 6, 1, 5, 7, 8, 2]


def _nepx():
    import nepx
    return nepx


def run_gpu(path, types, h, pos, pbc=(1, 1, 1), **kw):
    nepx = _nepx()
    pot = nepx.Potential(path, max_atoms=len(types))
    t = torch.as_tensor(np.asarray(types, dtype=np.int32), device="cuda")
    p = torch.as_tensor(np.ascontiguousarray(np.asarray(pos, dtype=np.float64)), device="cuda")
    pe, f, w = pot.compute(t, np.asarray(h, dtype=np.float64), p, pbc=pbc, sync_check=True, **kw)
    torch.cuda.synchronize()
    return pot, pe.cpu().numpy(), f.cpu().numpy(), w.cpu().numpy()


def assert_close(ref, got, label=""):
    pe0, f0, w0 = ref
    pe1, f1, w1 = got
    n = len(pe0)
    rel_f = np.linalg.norm(f1 - f0) / max(np.linalg.norm(f0), 1e-12)
    assert rel_f <= 2e-5, "%s force rel err %g" % (label, rel_f)
    assert np.all(np.abs(f1 - f0) <= 1e-4 * (1 + np.abs(f0))), label
    assert np.all(np.abs(pe1 - pe0) <= 2e-5 + 2e-6 * np.abs(pe0)), \
        "%s max dE %g" % (label, np.abs(pe1 - pe0).max())
    assert abs(pe1.sum() - pe0.sum()) / n <= 2e-6 + 2e-7 * abs(pe0.sum()) / n, label
    rel_w = np.linalg.norm(w1 - w0) / max(np.linalg.norm(w0), 1e-12)
    assert rel_w <= 5e-5, "%s virial rel err %g" % (label, rel_w)


@pytest.mark.parametrize("case", ["single_large_nve", "multi_nvt_restart", "nep_zbl_boundary"])
def test_golden_large_box(goldens, case):
    rec = goldens["static"][case]
    path = potential(rec["potential"])
    pos = np.array(rec["pos"]).T
    ref = oracle.OracleModel(path).compute(rec["type"], rec["h"], pos, rec["pbc"])
    _, pe, f, w = run_gpu(path, rec["type"], rec["h"], pos, rec["pbc"])
    assert_close(ref, (pe, f, w), case)
    # and the GPUMD golden itself, at the reference suite's tolerances
    fg = np.array(rec["force"]).T
    assert np.all(np.abs(f - fg) <= 1e-6 + 1e-4 * np.abs(fg))
    eg = np.array(rec["energy_atom"])
    assert np.all(np.abs(pe - eg) <= 1e-8 + 1e-5 * np.abs(eg) + 2e-5)
    wg = np.array(rec["virial_rowmajor"]).T
    assert np.all(np.abs(w[ROWMAJOR] - wg) <= 1e-6 + 1e-4 * np.abs(wg) + 2e-5)


def _water_box(n_mol, seed):
    t, h, p = workloads.water(n_mol=n_mol, seed=seed)
    return t, h, p


def test_water_model_random_box():
    t, h, p = _water_box(700, 1)            # 2100 atoms, L ~ 27.6 A
    path = potential("nep_water.txt")
    ref = oracle.OracleModel(path).compute(t, h, p)
    _, pe, f, w = run_gpu(path, t, h, p)
    assert_close(ref, (pe, f, w), "water")


def test_carbon_model_diamond():
    t, h, p = workloads.diamond(ncell=6, jitter=0.08, seed=2)   # 1728 atoms
    path = potential("nep_C.txt")
    ref = oracle.OracleModel(path).compute(t, h, p)
    _, pe, f, w = run_gpu(path, t, h, p)
    assert_close(ref, (pe, f, w), "carbon")


def test_triclinic_box():
    rng = np.random.default_rng(5)
    n = 600
    H = np.array([[19.0, 2.5, 1.2], [0.0, 18.5, 1.9], [0.0, 0.0, 19.2]])
    frac = rng.uniform(0, 1, (3, n))
    p = H @ frac
    t = rng.integers(0, 2, n).astype(np.int32)
    path = potential("nep_water.txt")
    ref = oracle.OracleModel(path).compute(t, H.reshape(-1), p)
    _, pe, f, w = run_gpu(path, t, H.reshape(-1), p)
    assert_close(ref, (pe, f, w), "triclinic")


@pytest.mark.parametrize("version,zbl", [(5, None), (4, (1.0, 2.0)), (5, (0.8, 1.6, 0.7)),
                                         (4, "flexible"), (5, "flexible")])
def test_synthetic_multitype(tmp_path, version, zbl):
    syms = ("C", "H", "O", "Cu")
    path = workloads.write_nep(str(tmp_path / "nep.txt"), version=version, symbols=syms, zbl=zbl,
                               rc=(5.0, 4.0), mn=(120, 60), H=24, seed=11, std=0.1)
    t, h, p = workloads.random_packed(900, 4, density=0.08, seed=3)
    ref = oracle.OracleModel(path).compute(t, h, p)
    _, pe, f, w = run_gpu(path, t, h, p)
    assert_close(ref, (pe, f, w), "nep%d zbl=%s" % (version, zbl))


@pytest.mark.parametrize("box", ["large", "small"])
def test_typewise_cutoffs(tmp_path, box):
    """Per-type cutoffs against the oracle, on the large-box and the small-box path."""
    path = workloads.write_nep(str(tmp_path / "nep.txt"), version=5, symbols=("O", "H"),
                               rc=((6.0, 4.0), (5.0, 3.5)), mn=(250, 100), l_max=(4, 2, 1),
                               H=20, seed=31, q_scaler=0.1)
    t, h, p = workloads.water(n_mol=400 if box == "large" else 30, seed=37)
    ref = oracle.OracleModel(path).compute(t, h, p)
    _, pe, f, w = run_gpu(path, t, h, p)
    assert_close(ref, (pe, f, w), "typewise cutoffs, %s box" % box)


def test_all_many_body_invariants(tmp_path):
    """l_max line with q_222, q_1111, q_112, q_123, q_233 and q_134 all on."""
    path = str(tmp_path / "nep_inv.txt")
    workloads.write_nep(path, version=4, symbols=("C", "O"), rc=(4.6, 4.0), mn=(90, 60),
                        l_max=(4, 2, 1), H=16, seed=7, std=0.1)
    lines = open(path).read().splitlines()
    # switch on the four optional invariants and extend the parameter block
    lines[4] = "l_max 4 1 1 1 1 1 1"
    T, nR, nA, kR, kA, H = 2, 5, 5, 9, 9, 16
    dim = nR + nA * (4 + 6)
    num = (dim + 2) * H * T + 1 + T * T * (nR * kR + nA * kA)
    rng = np.random.default_rng(9)
    body = ["%.8e" % v for v in rng.normal(0, 0.1, num)] + ["1.0"] * dim
    open(path, "w").write("\n".join(lines[:6] + body) + "\n")
    t, h, p = workloads.random_packed(700, 2, density=0.09, seed=4)
    ref = oracle.OracleModel(path).compute(t, h, p)
    _, pe, f, w = run_gpu(path, t, h, p)
    assert_close(ref, (pe, f, w), "invariants")


def test_neighbor_sets_match_fp32_predicate():
    t, h, p = _water_box(600, 3)
    path = potential("nep_water.txt")
    pot, _, _, _ = run_gpu(path, t, h, p)
    om = oracle.OracleModel(path)
    for which in (0, 1):
        got = pot.neighbors(which, len(t))
        want = om.neighbors_f32(t, h, p, which)
        rc = om.rc_radial if which == 0 else om.rc_angular
        for i in range(len(t)):
            a, b = set(got[i].tolist()), set(want[i].tolist())
            assert np.all(np.diff(got[i]) > 0), "row %d not ascending" % i
            for j in a ^ b:
                d = p[:, j] - p[:, i]
                d -= np.round(d / h[0]) * h[0]
                r = 0.5 * (rc[t[i]] + rc[t[j]])
                assert abs(d @ d - r * r) <= 4 * np.spacing(np.float32(r * r)), (i, j)


def test_deterministic_and_accumulate():
    t, h, p = _water_box(400, 4)
    path = potential("nep_water.txt")
    nepx = _nepx()
    pot = nepx.Potential(path, max_atoms=len(t))
    tt = torch.as_tensor(t, device="cuda")
    pp = torch.as_tensor(p, device="cuda")
    a = [x.clone() for x in pot.compute(tt, h, pp, sync_check=True)]
    b = [x.clone() for x in pot.compute(tt, h, pp, sync_check=True)]
    for x, y in zip(a, b):
        assert torch.equal(x, y), "results differ between identical calls"
    pot.compute(tt, h, pp, out=b, accumulate=True, sync_check=True)
    for x, y in zip(a, b):
        assert torch.allclose(2 * x, y, rtol=0, atol=1e-12)


def test_row_overflow_is_reported(tmp_path):
    """A too-small MN_angular is reported as NEPX_ERR_OVERFLOW, not a fault."""
    path = workloads.write_nep(str(tmp_path / "tiny.txt"), symbols=("O", "H"), rc=(6.0, 4.0),
                               mn=(150, 4), n_max=(4, 4), l_max=(4, 2, 0), H=8, seed=1)
    t, h, p = _water_box(300, 5)
    nepx = _nepx()
    with pytest.raises(nepx.NepxError) as err:
        run_gpu(path, t, h, p)
    assert err.value.code == 6


def test_capacity_and_box_errors():
    nepx = _nepx()
    t, h, p = _water_box(100, 6)
    pot = nepx.Potential(potential("nep_water.txt"), max_atoms=100)
    tt = torch.as_tensor(t, device="cuda")
    pp = torch.as_tensor(p, device="cuda")
    with pytest.raises(nepx.NepxError) as err:
        pot.compute(tt, h, pp)
    assert err.value.code == 5
