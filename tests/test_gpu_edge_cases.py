"""Edge cases of the force call: empty and one-atom inputs, atoms with no
neighbour, open and mixed boundaries, and the full-size workloads (1.0 M Cu
with ZBL, 8.0 M diamond C) through size-independent properties: forces sum
to zero, and a rigid translation of every atom changes neither the energy
nor any atom's force beyond FP32 rounding.
"""
import numpy as np
import pytest

import oracle
import workloads
from conftest import potential
from test_gpu_force import assert_close, run_gpu

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_empty_inputs_are_rejected():
    import nepx
    pot = nepx.Potential(potential("nep_C.txt"), max_atoms=8)
    t = torch.zeros(0, dtype=torch.int32, device="cuda")
    p = torch.zeros(3, 0, dtype=torch.float64, device="cuda")
    h = np.array([10.0, 0, 0, 0, 10.0, 0, 0, 0, 10.0])
    with pytest.raises(nepx.NepxError) as err:
        pot.compute(t, h, p)
    assert err.value.code == 1
    t1 = torch.zeros(4, dtype=torch.int32, device="cuda")
    p1 = torch.rand(3, 4, dtype=torch.float64, device="cuda") * 10.0
    with pytest.raises(nepx.NepxError) as err:
        pot.compute_batch([(4, h, (1, 1, 1)), (0, h, (1, 1, 1))], t1, p1)
    assert err.value.code == 1


def test_isolated_atoms():
    """Atoms farther apart than every cutoff: empty rows, zero force, the
    ANN energy of a zero descriptor."""
    rng = np.random.default_rng(3)
    n = 12
    grid = np.stack(np.meshgrid(np.arange(3), np.arange(2), np.arange(2), indexing="ij"), -1)
    pos = (grid.reshape(-1, 3)[:n] * 12.0 + 5.0 + rng.uniform(-0.5, 0.5, (n, 3))).T.copy()
    h = [40.0, 0, 0, 0, 40.0, 0, 0, 0, 40.0]
    t = rng.integers(0, 2, n)
    path = potential("nep_water.txt")
    ref = oracle.OracleModel(path).compute(t, h, pos)
    _, pe, f, w = run_gpu(path, t, h, pos)
    assert np.all(f == 0.0) and np.all(w == 0.0)
    assert np.allclose(pe, ref[0], rtol=1e-6, atol=1e-7)
    for k in (0, 1):   # one energy per type
        assert np.ptp(pe[t == k]) < 1e-7


@pytest.mark.parametrize("n", [1, 2, 3])
def test_few_atoms_in_a_small_cell(n):
    """One to three atoms in a periodic cell thinner than the cutoff: every
    neighbour is a periodic image (small-box path), including an atom's own."""
    rng = np.random.default_rng(n)
    H = np.array([[3.567, 0.3, 0.0], [0.0, 3.4, 0.2], [0.0, 0.0, 3.9]])
    pos = H @ rng.uniform(0, 1, (3, n))
    t = np.zeros(n, dtype=np.int32)
    path = potential("nep_C.txt")
    pe0, f0, w0 = oracle.OracleModel(path).compute(t, H.reshape(-1), pos)
    _, pe, f, w = run_gpu(path, t, H.reshape(-1), pos)
    # image contributions cancel (exactly, for one atom): FP32 sums leave
    # ~1e-6 eV/A, so forces get an absolute floor
    assert np.all(np.abs(f - f0) <= 1e-5 + 2e-5 * np.abs(f0)), (f, f0)
    assert np.all(np.abs(pe - pe0) <= 2e-5 + 2e-6 * np.abs(pe0))
    assert np.linalg.norm(w - w0) / np.linalg.norm(w0) <= 5e-5


@pytest.mark.parametrize("pbc", [(0, 0, 0), (1, 0, 0), (0, 1, 1)])
def test_open_and_mixed_boundaries(pbc):
    t, h, p = workloads.water(n_mol=400, seed=31)   # ~22.9 A: large box where periodic
    path = potential("nep_water.txt")
    ref = oracle.OracleModel(path).compute(t, h, p, pbc)
    _, pe, f, w = run_gpu(path, t, h, p, pbc=pbc)
    assert_close(ref, (pe, f, w), "pbc %s" % (pbc,))


def _invariants(path, t, h, p, shift):
    import nepx
    n = len(t)
    pot = nepx.Potential(path, max_atoms=n)
    tt = torch.as_tensor(np.asarray(t, dtype=np.int32), device="cuda")
    L = np.diag(np.asarray(h).reshape(3, 3))
    out = []
    for s in (np.zeros(3), shift):
        ps = torch.as_tensor(np.ascontiguousarray((p + s[:, None]) % L[:, None]), device="cuda")
        pe, f, _ = pot.compute(tt, h, ps, sync_check=True)
        out.append((pe.sum().item(), f))
        del ps
    (e0, f0), (e1, f1) = out
    fsum = f0.sum(dim=1).abs().max().item()
    fabs = f0.abs().sum(dim=1).max().item()
    assert fsum <= 1e-6 * fabs, (fsum, fabs)
    assert abs(e1 - e0) <= 1e-6 * abs(e0) + 1e-6 * n ** 0.5, (e0, e1)
    # per component: most atoms of a near-perfect crystal feel almost no
    # force, so FP32 rounding (~1e-6 eV/A) sets an absolute floor
    worst = ((f1 - f0).abs() - 2e-5 * f0.abs()).max().item()
    assert worst <= 2e-5, worst
    pot.close()


def test_full_size_copper_1m(tmp_path):
    """The 1.0 M-atom Cu workload (NEP-ZBL, 1% vacancies)."""
    path = workloads.write_nep(str(tmp_path / "cu.txt"), version=4, symbols=("Cu",),
                               zbl=(1.0, 2.0), rc=(5.0, 4.0), mn=(100, 60), n_max=(4, 4),
                               basis=(8, 8), l_max=(4, 2, 1), H=40, seed=2026, q_scaler=0.02)
    t, h, p = workloads.fcc(a=3.615, ncell=63, vacancy=0.01, seed=1)
    assert len(t) > 990000
    _invariants(path, t, h, p, np.array([1.37, -2.11, 0.53]))


def test_full_size_carbon_8m(tmp_path):
    """The 8.0 M-atom diamond workload with 10% displaced atoms."""
    path = workloads.write_nep(str(tmp_path / "c.txt"), version=4, symbols=("C",),
                               rc=(4.2, 3.7), mn=(100, 60), n_max=(4, 4), basis=(8, 8),
                               l_max=(4, 2, 1), H=30, seed=2025, q_scaler=0.02)
    t, h, p = workloads.diamond(a=3.567, ncell=100, jitter=0.05, seed=1)
    rng = np.random.default_rng(101)
    pick = rng.random(len(t)) < 0.10
    p[:, pick] = (p[:, pick] + rng.normal(0.0, 0.3, (3, int(pick.sum())))) % h[0]
    assert len(t) == 8000000
    _invariants(path, t, h, p, np.array([0.91, 0.37, -1.73]))
