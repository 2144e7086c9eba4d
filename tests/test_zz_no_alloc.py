"""nepx_compute_noalloc: the force call for callers that cannot allocate.

Some callers cannot call cudaMalloc while they run (their start-up hands all
device memory to their own pool allocator, or their rules forbid allocator
calls after initialisation).  nepx_compute_noalloc serves them from a 16 MiB
static device array inside the library.  This test drives it through the C
ABI and checks two calls in a row against the allocating nepx_compute on
the same inputs, at the force/energy/virial tolerance of the other GPU tests
(both paths run the same kernels, so they agree far inside it).  The file is
named to be collected last.
"""
import ctypes

import numpy as np
import pytest

import workloads
from conftest import potential

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _close(a, b):
    pe0, f0, w0 = [x.cpu().numpy() for x in a]
    pe1, f1, w1 = [x.cpu().numpy() for x in b]
    assert np.linalg.norm(f1 - f0) / np.linalg.norm(f0) <= 2e-5
    assert np.all(np.abs(pe1 - pe0) <= 2e-5 + 2e-6 * np.abs(pe0))
    assert np.linalg.norm(w1 - w0) / np.linalg.norm(w0) <= 5e-5


def test_noalloc_matches_allocating_path_twice():
    import nepx
    t, h, p = workloads.water(n_mol=600, seed=11)          # 1800 atoms
    n = len(t)
    # a handle sized for one atom: the no-alloc call needs no per-atom buffers from it
    pot_small = nepx.Potential(potential("nep_water.txt"), max_atoms=1)
    pot_full = nepx.Potential(potential("nep_water.txt"), max_atoms=n)
    tt = torch.as_tensor(t, device="cuda")
    pp = torch.as_tensor(p, device="cuda")
    ref = [x.clone() for x in pot_full.compute(tt, h, pp, sync_check=True)]
    box = nepx.make_box(h)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        out = [torch.full((n,), np.nan, dtype=torch.float64, device="cuda"),
               torch.full((3, n), np.nan, dtype=torch.float64, device="cuda"),
               torch.full((9, n), np.nan, dtype=torch.float64, device="cuda")]
        rc = nepx.lib().nepx_compute_noalloc(
            pot_small._h, ctypes.byref(box), n, ctypes.c_void_p(tt.data_ptr()),
            ctypes.c_void_p(pp.data_ptr()), ctypes.c_void_p(out[0].data_ptr()),
            ctypes.c_void_p(out[1].data_ptr()), ctypes.c_void_p(out[2].data_ptr()),
            ctypes.c_void_p(stream))
        assert rc == 0, nepx.lib().nepx_last_error(pot_small._h)
        torch.cuda.synchronize()
        _close(ref, out)


def test_noalloc_rejects_oversize_systems():
    import nepx
    t, h, p = workloads.water(n_mol=4000, seed=12)         # 12000 atoms: beyond 16 MiB
    pot = nepx.Potential(potential("nep_water.txt"), max_atoms=1)
    tt = torch.as_tensor(t, device="cuda")
    pp = torch.as_tensor(p, device="cuda")
    n = len(t)
    out = [torch.empty(n, dtype=torch.float64, device="cuda"),
           torch.empty(3, n, dtype=torch.float64, device="cuda"),
           torch.empty(9, n, dtype=torch.float64, device="cuda")]
    rc = nepx.lib().nepx_compute_noalloc(
        pot._h, ctypes.byref(nepx.make_box(h)), n, ctypes.c_void_p(tt.data_ptr()),
        ctypes.c_void_p(pp.data_ptr()), *[ctypes.c_void_p(x.data_ptr()) for x in out], None)
    assert rc == 5
