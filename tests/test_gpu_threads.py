"""Handles are independent: several host threads that each create a handle
and evaluate forces at the same time get the results of a single-threaded
call (per-handle scratch; process-wide tables set up once per device under a
lock).  Each handle autotunes its own lane grouping, so sums may run in
another lane order: agreement is to FP32 rounding, not bitwise."""
import threading

import numpy as np
import pytest

import workloads
from conftest import potential

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_concurrent_handles_match_single_thread():
    import nepx
    path = potential("nep_water.txt")
    t, h, p = workloads.water(n_mol=600, seed=41)
    tt = torch.as_tensor(np.asarray(t, dtype=np.int32), device="cuda")
    pp = torch.as_tensor(np.ascontiguousarray(p), device="cuda")
    ref = nepx.Potential(path, max_atoms=len(t))
    want = [x.cpu().numpy() for x in ref.compute(tt, h, pp, sync_check=True)]
    results, errors = {}, []

    def work(k):
        try:
            pot = nepx.Potential(path, max_atoms=len(t))
            for _ in range(3):
                got = [x.cpu().numpy() for x in pot.compute(tt, h, pp, sync_check=True)]
            results[k] = got
            pot.close()
        except Exception as exc:   # reported below
            errors.append(exc)

    threads = [threading.Thread(target=work, args=(k,)) for k in range(4)]
    for th in threads:
        th.start()
    for th in threads:
        th.join(timeout=120)
    assert not errors, errors
    assert len(results) == 4
    for pe, f, w in results.values():
        assert np.linalg.norm(f - want[1]) / np.linalg.norm(want[1]) < 1e-6
        assert np.abs(pe - want[0]).max() < 1e-5
        assert np.linalg.norm(w - want[2]) / np.linalg.norm(want[2]) < 1e-5
