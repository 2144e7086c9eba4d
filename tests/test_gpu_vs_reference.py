"""Parity with the reference's OWN FP32 GPU NEP evaluation.

oracle/_ref/libnep_ref_gpu.so is DMG-MD's src/gpumd_compat (GPUMD-derived
kernels) compiled for sm_100a from its sources.  The engine's plain-FP32
path must match it within 1e-5 relative force error (2-norm over all
components) and 1e-6 eV/atom in total energy, and its typewise neighbour
rows must be identical (same FP32 predicate, same ascending order).
Inputs stay far below the reference's MN capacities: its legacy kernels do
not guard row overflow.
"""
import os

import numpy as np
import pytest

import oracle
import workloads
from conftest import potential

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.ref_gpu_available(),
                                 reason="reference GPU library not built")]


def _both(path, t, h, p, tmp_path):
    import nepx
    cwd = os.getcwd()
    os.chdir(tmp_path)   # the reference appends neighbor.out to the working directory
    try:
        n = len(t)
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
        return ref, pot, [x.cpu().numpy() for x in out_r], [x.cpu().numpy() for x in out_m]
    finally:
        os.chdir(cwd)


@pytest.mark.parametrize("kind", ["water", "carbon"])
def test_force_energy_virial_match_reference_fp32(kind, tmp_path):
    if kind == "water":
        t, h, p = workloads.water(n_mol=1000, seed=7)
        path = potential("nep_water.txt")
    else:
        t, h, p = workloads.diamond(ncell=6, jitter=0.1, seed=8)
        path = potential("nep_C.txt")
    _, _, (pe0, f0, w0), (pe1, f1, w1) = _both(path, t, h, p, tmp_path)
    n = len(t)
    rel_f = np.linalg.norm(f1 - f0) / np.linalg.norm(f0)
    assert rel_f <= 1e-5, rel_f
    assert abs(pe1.sum() - pe0.sum()) / n <= 1e-6
    assert np.abs(pe1 - pe0).max() <= 2e-5
    assert np.linalg.norm(w1 - w0) / np.linalg.norm(w0) <= 2e-5


def test_neighbor_rows_bit_exact(tmp_path):
    t, h, p = workloads.water(n_mol=900, seed=9)
    path = potential("nep_water.txt")
    ref, pot, _, _ = _both(path, t, h, p, tmp_path)
    for which, mn in ((0, pot.info["MN_r"]), (1, pot.info["MN_a"])):
        a = ref.neighbors(which, mn)
        b = pot.neighbors(which, len(t))
        for i in range(len(t)):
            assert np.array_equal(a[i], b[i]), (which, i)


def _perovskite(ncell=8, a=4.0, jitter=0.05, seed=0):
    """BaTiO3 perovskite supercell: types Ba 0, Ti 1, O 2."""
    base = np.array([[0, 0, 0], [.5, .5, .5], [.5, .5, 0], [.5, 0, .5], [0, .5, .5]])
    kinds = np.array([0, 1, 2, 2, 2], dtype=np.int32)
    g = np.stack(np.meshgrid(*[np.arange(ncell)] * 3, indexing="ij"), -1).reshape(-1, 3)
    frac = (g[:, None, :] + base[None, :, :]).reshape(-1, 3) / ncell
    L = a * ncell
    rng = np.random.default_rng(seed)
    pos = (frac * L + rng.normal(0.0, jitter, frac.shape)) % L
    t = np.tile(kinds, len(g))
    return t, np.array([L, 0, 0, 0, L, 0, 0, 0, L], dtype=np.float64), np.ascontiguousarray(pos.T)


@pytest.mark.parametrize("case", ["nep5_four_types", "zbl_universal", "zbl_typewise",
                                  "zbl_flexible", "batio3_nep_zbl"])
def test_more_models_match_reference_fp32(case, tmp_path):
    """NEP5 with four types, NEP4-ZBL with the universal, the typewise and the
    flexible (fitted per-pair) ZBL (close contacts down to 0.9 A), and the
    reference suite's BaTiO3 NEP-ZBL potential on a perovskite supercell."""
    syms = ("C", "H", "O", "Cu")
    if case == "batio3_nep_zbl":
        path = potential("nep_BaTiO3_zbl.txt")
        t, h, p = _perovskite(seed=3)
    else:
        zbl = {"nep5_four_types": None, "zbl_universal": (1.0, 2.0),
               "zbl_typewise": (1.0, 2.0, 0.7), "zbl_flexible": "flexible"}[case]
        path = workloads.write_nep(str(tmp_path / "nep.txt"), version=5 if zbl is None else 4,
                                   symbols=syms, zbl=zbl, rc=(5.0, 4.0), mn=(160, 80),
                                   l_max=(4, 2, 1), H=32, seed=17, q_scaler=0.1)
        t, h, p = workloads.random_packed(n=2000, num_types=4, density=0.08, seed=19)
    _, _, (pe0, f0, w0), (pe1, f1, w1) = _both(path, t, h, p, tmp_path)
    n = len(t)
    rel_f = np.linalg.norm(f1 - f0) / np.linalg.norm(f0)
    assert rel_f <= 1e-5, rel_f
    assert abs(pe1.sum() - pe0.sum()) / n <= 1e-6
    assert np.abs(pe1 - pe0).max() <= 2e-5
    assert np.linalg.norm(w1 - w0) / np.linalg.norm(w0) <= 2e-5


def test_typewise_cutoffs_match_reference(tmp_path):
    """Per-type cutoffs (O 6.0/4.0 A, H 5.0/3.5 A; a pair uses the mean of
    its two types' cutoffs, nep.cu:503-561): forces and energies within the
    FP32 tolerances and typewise rows identical to the reference's."""
    path = workloads.write_nep(str(tmp_path / "nep.txt"), version=4, symbols=("O", "H"),
                               rc=((6.0, 4.0), (5.0, 3.5)), mn=(250, 100), l_max=(4, 2, 0),
                               H=30, seed=23, q_scaler=0.1)
    t, h, p = workloads.water(n_mol=900, seed=29)
    ref, pot, (pe0, f0, w0), (pe1, f1, w1) = _both(path, t, h, p, tmp_path)
    n = len(t)
    assert np.linalg.norm(f1 - f0) / np.linalg.norm(f0) <= 1e-5
    assert abs(pe1.sum() - pe0.sum()) / n <= 1e-6
    assert np.linalg.norm(w1 - w0) / np.linalg.norm(w0) <= 2e-5
    for which, mn in ((0, pot.info["MN_r"]), (1, pot.info["MN_a"])):
        a = ref.neighbors(which, mn)
        b = pot.neighbors(which, n)
        for i in range(n):
            assert np.array_equal(a[i], b[i]), (which, i)


def test_all_many_body_invariants_match_reference(tmp_path):
    """q_222, q_1111, q_112, q_123, q_233 and q_134 all on: the engine's and the
    oracle's monomial tables of these invariants are both transcriptions of
    find_q (nep_utilities.cuh:1602-1730), so the reference's own kernels are
    the independent check."""
    path = workloads.write_nep(str(tmp_path / "nep.txt"), version=4, symbols=("C", "O"),
                               rc=(4.6, 4.0), mn=(90, 60), l_max=(4, 1, 1, 1, 1, 1, 1), H=16,
                               seed=41, q_scaler=0.1)
    t, h, p = workloads.random_packed(2000, 2, density=0.09, seed=43)
    _, _, (pe0, f0, w0), (pe1, f1, w1) = _both(path, t, h, p, tmp_path)
    n = len(t)
    assert np.linalg.norm(f1 - f0) / np.linalg.norm(f0) <= 1e-5
    assert abs(pe1.sum() - pe0.sum()) / n <= 1e-6
    assert np.abs(pe1 - pe0).max() <= 2e-5
    assert np.linalg.norm(w1 - w0) / np.linalg.norm(w0) <= 2e-5

