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
