"""Batched evaluation and the continuous-batching server.

* nepx_compute_batch on a mix of small and large boxes of different sizes
  equals the FP64 oracle per structure (tolerances of test_gpu_force.py),
  equals a batch of that structure alone bit for bit, and equals
  nepx_compute on the structure within FP32 rounding (1e-6 relative force,
  1e-5 eV per atom: the Verlet path sums the same edges in another lane
  order);
* the server returns, for every request of a randomly ordered stream that
  overflows its arena several times, exactly the batch-of-one result;
* an MD segment run by the server follows nepx_md's NVE trajectory;
* a server sized from a device-memory budget admits by bytes.
"""
import numpy as np
import pytest

import oracle
import workloads
from conftest import potential
from test_gpu_force import assert_close

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

WATER = "nep_water.txt"


def _structures(seed=0):
    rng = np.random.default_rng(seed)
    out = []
    t, h, p = workloads.water(n_mol=30, seed=1)              # small box, 90 atoms
    out.append((t, h, p, (1, 1, 1)))
    t, h, p = workloads.water(n_mol=300, seed=2)             # large box, 900 atoms
    out.append((t, h, p, (1, 1, 1)))
    t, h, p = workloads.random_packed(n=24, num_types=2, density=0.08, seed=3)
    out.append((t, h, p, (1, 1, 1)))                         # tiny, many images
    t, h, p = workloads.water(n_mol=40, seed=4)              # slab, z not periodic
    h = (np.array(h).reshape(3, 3) * np.diag([1.0, 1.0, 2.5])).reshape(-1)
    out.append((t, h, p, (1, 1, 0)))
    t, h, p = workloads.water(n_mol=220, seed=5)             # large box, 660 atoms
    out.append((t, h, p, (1, 1, 1)))
    order = rng.permutation(len(out))
    return [out[k] for k in order]


def _pack(structs):
    t = np.concatenate([np.asarray(s[0], dtype=np.int32) for s in structs])
    p = np.concatenate([np.asarray(s[2], dtype=np.float64) for s in structs], axis=1)
    descs = [(len(s[0]), s[1], s[3]) for s in structs]
    return (torch.as_tensor(t, device="cuda"),
            torch.as_tensor(np.ascontiguousarray(p), device="cuda"), descs)


def _split(arr, structs):
    out, o = [], 0
    for s in structs:
        n = len(s[0])
        out.append(arr[..., o:o + n])
        o += n
    return out


def _batch_one(pot, s):
    tt, pp, descs = _pack([s])
    pe, f, w = pot.compute_batch(descs, tt, pp, sync_check=True)
    return pe.cpu().numpy(), f.cpu().numpy(), w.cpu().numpy()


def test_batch_matches_oracle_and_single():
    import nepx
    structs = _structures()
    total = sum(len(s[0]) for s in structs)
    pot = nepx.Potential(potential(WATER), max_atoms=total)
    tt, pp, descs = _pack(structs)
    pe, f, w = pot.compute_batch(descs, tt, pp, sync_check=True)
    pe, f, w = pe.cpu().numpy(), f.cpu().numpy(), w.cpu().numpy()
    orc = oracle.OracleModel(potential(WATER))
    for k, (s, pe_k, f_k, w_k) in enumerate(zip(structs, _split(pe, structs), _split(f, structs),
                                                 _split(w, structs))):
        t, h, p, pbc = s
        assert_close(orc.compute(t, h, p, pbc), (pe_k, f_k, w_k), "struct %d" % k)
        one = _batch_one(pot, s)
        assert np.array_equal(one[0], pe_k) and np.array_equal(one[1], f_k), k
        assert np.array_equal(one[2], w_k), k
        ts = torch.as_tensor(np.asarray(t, dtype=np.int32), device="cuda")
        ps = torch.as_tensor(np.ascontiguousarray(p), device="cuda")
        pe1, f1, w1 = pot.compute(ts, h, ps, pbc=pbc, sync_check=True)
        f1 = f1.cpu().numpy()
        # FP32 sums over the same edges in another lane order: rounding-level
        assert np.linalg.norm(f1 - f_k) / np.linalg.norm(f_k) < 1e-6, k
        assert np.abs(pe1.cpu().numpy() - pe_k).max() < 1e-5, k


def test_server_stream_equals_batch_of_one():
    import nepx
    rng = np.random.default_rng(7)
    base = _structures(seed=1)
    stream = [base[k] for k in rng.integers(0, len(base), 25)]
    pot = nepx.Potential(potential(WATER), max_atoms=2000)
    expected = [_batch_one(pot, s) for s in stream]
    srv = nepx.Server(pot, max_atoms=2000, max_struct=6)     # a few requests at a time
    tickets = [srv.submit(t, p, h, pbc) for (t, h, p, pbc) in stream]
    for tk, exp in zip(tickets, expected):
        r = srv.wait(tk)
        assert np.array_equal(r["pe"], exp[0])
        assert np.array_equal(r["force"], exp[1])
        assert np.array_equal(r["virial"], exp[2])
        assert r["t_submit"] <= r["t_admit"] <= r["t_done"]
    st = srv.stats()
    assert st["done"] == len(stream) and st["steps"] >= 4
    srv.close()


def test_server_md_segment_follows_nepx_md():
    import nepx
    t, h, p = workloads.diamond(ncell=2, jitter=0.03, seed=31)     # 64 atoms, small box
    masses = np.full(len(t), 12.011)
    v = workloads.maxwell_boltzmann(masses, 300.0, seed=32)
    pot = nepx.Potential(potential("nep_C.txt"), max_atoms=4096)
    md = nepx.MD(pot, t, masses, p, v, h)
    md.set_ensemble("nve")
    md.run(40, 0.5)
    ref = md.state()
    md.close()
    srv = nepx.Server(pot, max_atoms=4096, max_struct=8)
    # the segment shares the arena with single points that come and go
    t2, h2, p2 = workloads.diamond(ncell=3, jitter=0.05, seed=33)
    others = [srv.submit(t2, p2, h2) for _ in range(3)]
    tk = srv.submit(t, p, h, md_steps=40, dt_fs=0.5, masses=masses, vel=v, want_state=True)
    others += [srv.submit(t2, p2, h2) for _ in range(3)]
    r = srv.wait(tk)
    for o in others:
        srv.wait(o)
    np.testing.assert_allclose(r["pos"], ref["pos"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(r["vel"], ref["vel"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(r["force"], ref["force"], rtol=0, atol=1e-7)
    srv.close()


def test_server_admits_by_device_memory():
    """A server sized from a byte budget holds the resident requests' bytes
    to it (a few structures at a time here), returns every request's
    batch-of-one result, and rejects a request that alone exceeds it."""
    import nepx
    rng = np.random.default_rng(9)
    base = _structures(seed=2)
    stream = [base[k] for k in rng.integers(0, len(base), 16)]
    pot = nepx.Potential(potential(WATER), max_atoms=2000)
    expected = [_batch_one(pot, s) for s in stream]
    probe = nepx.Server(pot, max_atoms=2000, max_struct=8)
    per_atom = probe.memory()["bytes_per_atom"]
    probe.close()
    budget = 1400 * per_atom          # about two of the larger structures
    srv = nepx.Server(pot, max_struct=8, hbm_bytes=budget)
    mem = srv.memory()
    assert mem["budget_bytes"] == pytest.approx(budget, rel=1e-9)
    tickets = [srv.submit(t, p, h, pbc) for (t, h, p, pbc) in stream]
    for tk, exp in zip(tickets, expected):
        r = srv.wait(tk)
        assert np.array_equal(r["pe"], exp[0])
        assert np.array_equal(r["force"], exp[1])
    st, mem = srv.stats(), srv.memory()
    assert st["done"] == len(stream)
    assert 0 < mem["mean_resident_bytes"] <= budget
    t, h, p = workloads.water(n_mol=600, seed=8)            # 1800 atoms: over the budget
    with pytest.raises(nepx.NepxError) as err:
        srv.submit(t, p, h)
    assert err.value.code == 5
    srv.close()


def _md_stream(seed):
    """MD segments of water in small, large and slab boxes (300 K, 1 fs:
    the hydrogens pass skin / 2 within a few tens of steps) mixed with single
    points, in a random order."""
    rng = np.random.default_rng(seed)
    mass_of = np.array([15.999, 1.008])
    out = []
    for k, s in enumerate(_structures(seed=seed)):
        t, h, p, pbc = s
        m = mass_of[np.asarray(t)]
        v = workloads.maxwell_boltzmann(m, 300.0, seed=40 + k)
        out.append((t, h, p, pbc, 60, m, v))
        out.append((t, h, p, pbc, 0, None, None))
    return [out[k] for k in rng.permutation(len(out))]


def test_server_row_reuse_equals_fresh_rows():
    """MD segments that keep Verlet candidates and filter them into their
    rows at each step (rebuilding them when an atom has moved more than
    skin / 2) give bit for bit the results of segments whose rows are built
    afresh at every step; the candidates were rebuilt inside the segments and
    reused on most steps."""
    import nepx
    stream = _md_stream(3)
    pot = nepx.Potential(potential(WATER), max_atoms=4000)
    outs = []
    for reuse in (True, False):
        srv = nepx.Server(pot, max_atoms=4000, max_struct=8)
        srv.set_row_reuse(reuse)
        tickets = [srv.submit(t, p, h, pbc, md_steps=ms, dt_fs=1.0, masses=m, vel=v,
                              want_state=True)
                   for (t, h, p, pbc, ms, m, v) in stream]
        outs.append([srv.wait(tk) for tk in tickets])
        rows = srv.rows()
        if reuse:
            md_atoms = sum(len(s[0]) for s in stream if s[4])
            # every segment built its candidates once on admission; more builds
            # mean skin-triggered rebuilds, fewer than the kept centers reuse
            assert rows["builds"] > md_atoms, rows
            assert rows["builds"] < 0.5 * rows["kept"], rows
        else:
            assert rows["builds"] == 0 and rows["kept"] == 0, rows
        srv.close()
    for a, b in zip(*outs):
        for key in ("pe", "force", "virial", "pos", "vel"):
            assert np.array_equal(a[key], b[key]), key
