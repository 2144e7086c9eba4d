"""nepx_compute_noalloc: the force call for callers that cannot allocate.

Some callers cannot call cudaMalloc while they run: their start-up hands all
device memory to their own pool allocator, or their rules forbid allocator
calls after initialisation.  nepx_compute_noalloc serves them from a 16 MiB
static device array inside the library, shared by every call and keeping the
last call's contents.  These tests drive it through the C ABI:

  * two calls in a row against the allocating nepx_compute on the same inputs;
  * a sequence that leaves stale rows, cell counts and flags behind in the
    shared array -- a larger system, a smaller one in another box, a call
    whose rows overflow (NEPX_ERR_OVERFLOW), then a clean call -- with every
    successful result checked against the FP64 oracle at the tolerances of
    the other GPU parity tests (test_gpu_force.assert_close);
  * systems beyond the array's size are rejected with NEPX_ERR_CAPACITY.

The file is named to be collected last.
"""
import ctypes
import os
import tempfile

import numpy as np
import pytest

import oracle
import workloads
from conftest import potential
from test_gpu_force import assert_close

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _close(a, b):
    pe0, f0, w0 = [x.cpu().numpy() for x in a]
    pe1, f1, w1 = [x.cpu().numpy() for x in b]
    assert np.linalg.norm(f1 - f0) / np.linalg.norm(f0) <= 2e-5
    assert np.all(np.abs(pe1 - pe0) <= 2e-5 + 2e-6 * np.abs(pe0))
    assert np.linalg.norm(w1 - w0) / np.linalg.norm(w0) <= 5e-5


def _noalloc(pot, t, h, p):
    """One nepx_compute_noalloc call into NaN-filled outputs: (rc, pe, f, w)."""
    import nepx
    n = len(t)
    tt = torch.as_tensor(np.asarray(t, dtype=np.int32), device="cuda")
    pp = torch.as_tensor(np.ascontiguousarray(p, dtype=np.float64), device="cuda")
    out = [torch.full((n,), np.nan, dtype=torch.float64, device="cuda"),
           torch.full((3, n), np.nan, dtype=torch.float64, device="cuda"),
           torch.full((9, n), np.nan, dtype=torch.float64, device="cuda")]
    stream = torch.cuda.current_stream().cuda_stream
    rc = nepx.lib().nepx_compute_noalloc(
        pot._h, ctypes.byref(nepx.make_box(h)), n, ctypes.c_void_p(tt.data_ptr()),
        ctypes.c_void_p(pp.data_ptr()), *[ctypes.c_void_p(x.data_ptr()) for x in out],
        ctypes.c_void_p(stream))
    torch.cuda.synchronize()
    return rc, out


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
    for call in range(2):
        rc, out = _noalloc(pot_small, t, h, p)
        assert rc == 0, nepx.lib().nepx_last_error(pot_small._h)
        _close(ref, out)


def _tight_water_model():
    """The water potential with its radial row capacity cut to 20 (x1.25 = 25
    slots, and the Verlet rows sized from it: well below the ~90 radial and
    ~140 Verlet neighbours of liquid water)."""
    with open(potential("nep_water.txt")) as f:
        lines = f.read().splitlines()
    assert lines[1].startswith("cutoff")
    lines[1] = "cutoff 6.0 4.0 20 80"
    path = os.path.join(tempfile.mkdtemp(), "nep_water_tight.txt")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path


def test_noalloc_sequence_against_oracle():
    import nepx
    path = potential("nep_water.txt")
    pot = nepx.Potential(path, max_atoms=1)
    ref_model = oracle.OracleModel(path)
    big = workloads.water(n_mol=800, seed=21)              # 2400 atoms, L ~ 28.8 A
    small = workloads.water(n_mol=300, seed=22, density=0.9)   # 900 atoms, another box
    assert not np.allclose(np.asarray(big[1]), np.asarray(small[1]))
    for label, (t, h, p) in (("larger system", big), ("smaller system", small)):
        rc, out = _noalloc(pot, t, h, p)
        assert rc == 0, "%s: %s" % (label, nepx.lib().nepx_last_error(pot._h))
        got = [x.cpu().numpy() for x in out]
        assert_close(ref_model.compute(t, h, p), got, label)
    # a model whose radial rows are too short: the call reports the overflow
    tight = nepx.Potential(_tight_water_model(), max_atoms=1)
    rc, _ = _noalloc(tight, *small)
    assert rc == 6, "expected NEPX_ERR_OVERFLOW, got %d" % rc
    assert b"neighbour row exceeded" in nepx.lib().nepx_last_error(tight._h)
    # the next call on the shared array starts from cleared flags and fresh rows
    t, h, p = big
    rc, out = _noalloc(pot, t, h, p)
    assert rc == 0, nepx.lib().nepx_last_error(pot._h)
    assert_close(ref_model.compute(t, h, p), [x.cpu().numpy() for x in out], "clean call")


def test_noalloc_rejects_oversize_systems():
    import nepx
    t, h, p = workloads.water(n_mol=4000, seed=12)         # 12000 atoms: beyond 16 MiB
    pot = nepx.Potential(potential("nep_water.txt"), max_atoms=1)
    rc, _ = _noalloc(pot, t, h, p)
    assert rc == 5
