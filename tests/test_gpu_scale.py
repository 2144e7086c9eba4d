"""Parity at the sizes the benchmark quotes its throughput on.

* Large carbon (8,000,000 atoms, the benchmark's headline workload) and FCC
  copper with NEP-ZBL (1.0 M atoms): the FP32 path against
  - the reference's FP64 CPU evaluator NEP3_CPU on spherical clusters cut
    out of the system (core radius 12 A; a shell of 2 rc keeps every core
    atom's energy, force and virial equal to the full system's):
    test_gpu_force.assert_close tolerances plus force RMSE <= 1e-4 eV/A;
  - the reference's own FP32 GPU kernels on the whole system: relative
    force error (2-norm) <= 1e-5 and total energy <= 1e-6 eV/atom, the
    contract of tests/test_gpu_vs_reference.py;
  and the mixed-precision path against the same FP64 values: force RMSE
  <= 1e-4 eV/A (relative 2-norm <= 1e-2).
* The serving stream (one four-type NEP5 for all requests): every request
  of a sample, single points and NVE segments of uneven size, served by the
  continuous-batching server, against the FP64 oracle at its returned state.

The reference's legacy kernels do not guard neighbour-row overflow, so they
run only after the engine has shown every row (Verlet, radial, angular)
below its capacity on the same positions.
"""
import os

import numpy as np
import pytest

import oracle
import workloads
from test_gpu_force import assert_close

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

MIXED_RMSE = 1e-4       # eV/A, force RMSE of the mixed path against FP64
MIXED_REL = 1e-2        # relative 2-norm of the mixed path's force error


def _cutout_reference(path, t, h, p, rc_max, clusters, r_core, seed):
    """FP64 NEP3_CPU energies / forces / virials of the cores of `clusters`
    cut-outs around random atoms: (indices, pe, f, w)."""
    ref = oracle.RefCpuModel(path)
    rng = np.random.default_rng(seed)
    idx, pe, f, w = [], [], [], []
    for c in rng.choice(len(t), clusters, replace=False):
        tc, hc, pc, core, orig = workloads.cutout(t, h, p, int(c), r_core, 2 * rc_max + 0.1)
        pe_c, f_c, w_c = ref.compute(tc, hc, pc, threads=os.cpu_count() or 1)
        idx.append(orig)
        pe.append(pe_c[core])
        f.append(f_c[:, core])
        w.append(w_c[:, core])
    return (np.concatenate(idx), np.concatenate(pe), np.concatenate(f, axis=1),
            np.concatenate(w, axis=1))


def _at_scale(spec, t, h, p, tmp_path, clusters=4, r_core=12.0, seed=3):
    import nepx
    if not (oracle.ref_cpu_available() and oracle.ref_gpu_available()):
        pytest.skip("reference libraries (oracle/_ref) not built")
    path = workloads.write_nep(str(tmp_path / "nep.txt"), **spec)
    n = len(t)
    tt = torch.as_tensor(np.asarray(t, dtype=np.int32), device="cuda")
    pp = torch.as_tensor(np.ascontiguousarray(p, dtype=np.float64), device="cuda")
    pot = nepx.Potential(path, max_atoms=n)
    got32 = [x.cpu().numpy() for x in pot.compute(tt, h, pp, sync_check=True)]
    max_r, max_a, max_v = pot.neighbor_stats()
    pot.set_precision("mixed")
    gotm = [x.cpu().numpy() for x in pot.compute(tt, h, pp, sync_check=True)]
    info = dict(pot.info)
    pot.close()
    # every row inside its capacity: the reference's kernels may run here
    mn_v = int(info["MN_r"] * ((max(spec["rc"]) + 1.0) / max(spec["rc"])) ** 3)
    assert max_r <= info["MN_r"] and max_a <= info["MN_a"] and max_v <= mn_v, \
        (max_r, max_a, max_v)

    # FP64 on cut-outs
    idx, pe0, f0, w0 = _cutout_reference(path, t, h, p, max(spec["rc"]), clusters, r_core, seed)
    assert len(idx) > 1000
    pe1, f1, w1 = [x[..., idx] for x in got32]
    assert_close((pe0, f0, w0), (pe1, f1, w1), "fp32 vs NEP3_CPU")
    assert np.sqrt(np.mean((f1 - f0) ** 2)) <= 1e-4
    fm = gotm[1][:, idx]
    rmse_m = np.sqrt(np.mean((fm - f0) ** 2))
    rel_m = np.linalg.norm(fm - f0) / np.linalg.norm(f0)
    assert rmse_m <= MIXED_RMSE and rel_m <= MIXED_REL, (rmse_m, rel_m)

    # the reference's own FP32 GPU kernels on the whole system
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
        pe_r, f_r, _ = [x.cpu().numpy() for x in out_r]
        del ref, out_r
    finally:
        os.chdir(cwd)
    rel_f = np.linalg.norm(got32[1] - f_r) / np.linalg.norm(f_r)
    assert rel_f <= 1e-5, rel_f
    assert abs(got32[0].sum() - pe_r.sum()) / n <= 1e-6


def test_large_carbon_8m(tmp_path):
    """The benchmark's headline system: 8,000,000 atoms of diamond with a
    random 10% displaced by N(0, 0.3 A), synthetic NEP4 (rc 4.2/3.7 A)."""
    t, h, p = workloads.displaced_diamond(ncell=100, seed=1)
    assert len(t) == 8000000
    _at_scale(workloads.NEP_SPECS["carbon"], t, h, p, tmp_path)


def test_copper_nep_zbl_1m(tmp_path):
    """1,000,188-site FCC copper with 1% vacancies, synthetic NEP4-ZBL."""
    t, h, p = workloads.fcc(a=3.615, ncell=63, vacancy=0.01, jitter=0.05, seed=1)
    assert len(t) > 990000
    _at_scale(workloads.NEP_SPECS["copper"], t, h, p, tmp_path)


def test_serving_requests_against_oracle(tmp_path):
    """A sample of the serving stream (sizes 16..8192 atoms, diamond C, FCC
    Cu and random-packed C/H/O/Cu; some 100-step NVE segments) through the
    server, each result against the FP64 oracle at the request's returned
    state."""
    import nepx
    path = workloads.write_nep(str(tmp_path / "nep5.txt"), **workloads.NEP_SPECS["serving"])
    stream = workloads.serving_stream(30, seed=11, md_steps=20)
    assert any(r["md_steps"] for r in stream) and any(not r["md_steps"] for r in stream)
    pot = nepx.Potential(path, max_atoms=65536)
    srv = nepx.Server(pot, max_atoms=65536, max_struct=64)
    tickets = [srv.submit(r["type"], r["pos"], r["h"], md_steps=r["md_steps"], dt_fs=1.0,
                          masses=r["mass"], vel=r["vel"], want_state=True) for r in stream]
    results = [srv.wait(tk) for tk in tickets]
    srv.close()
    pot.close()
    model = oracle.OracleModel(path)
    for k, (r, res) in enumerate(zip(stream, results)):
        pos = res["pos"] if r["md_steps"] else r["pos"]
        if r["md_steps"]:
            assert not np.allclose(pos, r["pos"])            # the segment moved the atoms
        ref = model.compute(r["type"], r["h"], pos)
        assert_close(ref, (res["pe"], res["force"], res["virial"]),
                     "request %d (%d atoms, %d steps)" % (k, len(r["type"]), r["md_steps"]))
