#!/usr/bin/env python3
"""Benchmark of the nepx NEP molecular-dynamics engine on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload carbon8m|water|copper|carbon|serving]

Default workload (the headline): large carbon NVE -- 8,000,000 atoms, a
100x100x100-cell diamond supercell (a = 3.567 A, 8 atoms per cubic cell,
jitter N(0, 0.05 A)) with a random 10% of the atoms displaced by N(0, 0.3 A)
(amorphous regions); synthetic one-type NEP4 (rc 4.2/3.7 A, n_max 4/4, basis
8/8, l_max 4 2 1 with the 4- and 5-body invariants, 30 hidden units, weights
N(0, 0.1^2), seeded; a descriptor scale q_scaler = 0.02 keeps the
random-weight landscape gentle), Maxwell-Boltzmann velocities at 300 K, NVE,
dt 1 fs.  One "step" is one full MD step: skin check and conditional Verlet
rebuild, NEP energy/force/virial, FP64 velocity Verlet, thermo reduction.
Metric: atom-steps/s, whole job (sum over ranks).

value  -- device time (CUDA events on the MD stream) of K steps queued in
          chunks of `--chunk` steps, each chunk preceded by a 512 MiB write
          that flushes the 126 MB L2 (the system's positions alone are
          192 MB); max over ranks.
e2e    -- the same K steps driven through the public C API one step per call
          (nepx_md_run: graph launch, thermo row D2H, synchronisation), host
          wall clock.
roofline -- the force kernels (k_filter_radial, k_nep_fused, k_gather, and
          k_angular_f12 unless the autotuner moved the angular partial forces
          into k_nep_fused): the FP32 operations of the algorithm they run
          (flops_per_atom + gather_flops_per_atom, per atom at the system's
          mean neighbour counts) over their CUDA-event time, against the FP32
          FMA peak of B200 (148 SMs x 128 lanes x 2 FLOP x max SM clock).
          traffic: their DRAM bytes per force call from ncu.
cpu_baseline -- the reference's own FP64 CPU NEP evaluator (NEP3_CPU,
          oracle/_ref) on all host cores, on a bounded sample of the same
          workload (a periodic block of the same lattice, same displacement
          statistics, every atom a center): force call, and md_step with a
          CPU velocity-Verlet update around it.
err_vs_fp64 -- force RMSE and energy error of the FP32 and mixed paths on the
          final MD state against NEP3_CPU (FP64) on spherical clusters cut out
          of it (core atoms whose 2 rc neighbourhood is inside the cluster:
          their results equal the full system's).
mixed_precision -- the same MD with the ANN on the tcgen05 tensor cores.
other_workloads -- water (24,000 atoms, Bussi NVT) and copper (1.0 M atoms,
          NEP-ZBL, Berendsen NPT): MD rate, force call, mixed precision and
          FP64 errors.
nve_drift -- NVE energy drift (eV/atom/ns) of 4096-atom diamond carbon,
          both precisions: 20 ps from the lattice, and 200 ps after 10 ps of
          Berendsen NVT (slope, its block standard error, 20 ps sub-windows).
serving -- a 5,000-request sample of the serving stream (--workload serving
          runs the full 20,000): served structures/s, p50/p99 latency at 30,
          60 and 90% of saturation, batched engine over the plain FP32 path.

--impl reference times that same reference CPU evaluator (force call plus a
CPU velocity-Verlet update on the bounded sample, rank 0) on the same config
dict, and the reference's own GPU kernels (src/gpumd_compat built for
sm_100a) on the full system (reference_gpu).
Multi-GPU: one independent replica per GPU (the reference's one-rank path
does not shard; replicas only), no collective on the data path.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "dmg-md_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import numpy as np  # noqa: E402

import workloads  # noqa: E402

K_B = 8.617343e-5
# DRAM bytes per atom and force call of the force kernels (k_filter_radial,
# k_nep_fused with the angular partial forces inside, k_gather at four CTAs
# per SM: the builds the autotuner picks for this model), dram__bytes_read.sum
# + dram__bytes_write.sum of one ncu-captured launch each on the large-carbon
# system at 1,000,000 atoms (--ncell 50), divided by its atoms (traffic grows
# with the atoms processed).  Keyed by workload and the kernel list; another
# form reports no traffic.
TRAFFIC_PER_ATOM = {
    ("carbon8m", ("k_filter_radial", "k_nep_fused", "k_gather")):
        (701.6 + 412.2 + 349.1 + 567.1 + 1359.3 + 292.3) * 1e6 / 1.0e6}
FP32_LANES = 148 * 128          # B200: SMs x FP32 lanes
SM_MAX_MHZ = 1965.0
L2_NOTE = "flushed by a 512 MiB write before every %d-step chunk"

WORKLOADS = {
    # name: (builder, nep kwargs, ensemble kwargs, dt_fs)
    "water": dict(
        nep=workloads.NEP_SPECS["water"],
        ens=dict(kind="nvt_bdp", T0=300.0, Tdamp=100.0), dt=0.5, T=300.0,
        desc="water_8000mol_24000atoms_nep4_O-H_rc6.0-4.0_H50_nvt_bdp_300K_dt0.5fs"),
    "carbon": dict(
        nep=workloads.NEP_SPECS["carbon"],
        ens=dict(kind="nve"), dt=1.0, T=300.0,
        desc="diamond_8x8x8_4096atoms_nep4_C_rc4.2-3.7_H30_nve_dt1fs"),
    "copper": dict(
        nep=workloads.NEP_SPECS["copper"],
        ens=dict(kind="npt_ber", T0=300.0, Tdamp=100.0, p_gpa=0.0, bulk_gpa=140.0,
                 tau_p=1000.0), dt=1.0, T=300.0,
        desc="cu_fcc_63x63x63_1pct_vacancies_nepzbl_rc5.0-4.0_H40_npt_ber_dt1fs"),
}

WORKLOADS["carbon8m"] = dict(
    WORKLOADS["carbon"],
    desc="diamond_100x100x100cells_8000000atoms_10pct_displaced_nep4_C_rc4.2-3.7_H30_"
         "nve_300K_dt1fs")

MASSES = {"O": 15.999, "H": 1.008, "C": 12.011, "Cu": 63.546}

# serving stream: one shared synthetic four-type NEP5 (C, H, O, Cu)
SERVING_NEP = workloads.NEP_SPECS["serving"]


def _percentile_ms(xs, q):
    return float(np.percentile(np.asarray(xs) * 1e3, q)) if len(xs) else None


def run_serving(args):
    """Served structures/s (saturation) and p50/p99 latency (Poisson arrivals
    at 30, 60 and 90% of saturation) of the continuous-batching
    server on a stream of independent structures (log-uniform 16..8192
    atoms; diamond C, FCC Cu, random-packed C/H/O/Cu; a fifth of the
    requests are 100-step NVE segments at dt 1 fs), next to the same
    requests evaluated one at a time through the plain single-system path
    (nepx_compute / nepx_md per request, host buffers in and out)."""
    import torch
    import nepx
    count = args.requests
    stream = workloads.serving_stream(count, seed=11)
    tmp = tempfile.mkdtemp()
    path = workloads.write_nep(os.path.join(tmp, "nep.txt"), **SERVING_NEP)
    arena, slots = args.arena, 2048
    pot = nepx.Potential(path, max_atoms=arena)
    pot.set_precision(args.precision)
    work = [len(r["type"]) * (1 + r["md_steps"]) for r in stream]
    total_atom_steps = float(sum(work))

    def submit(srv, r):
        return srv.submit(r["type"], r["pos"], r["h"], md_steps=r["md_steps"], dt_fs=1.0,
                          masses=r["mass"], vel=r["vel"], want_virial=False)

    # warm-up: autotune and first-touch of the arena
    srv = nepx.Server(pot, max_atoms=arena, max_struct=slots)
    for r in stream[:8]:
        srv.wait(submit(srv, dict(r, md_steps=0, mass=None, vel=None)))
    srv.close()
    def new_server():
        srv = nepx.Server(pot, max_atoms=arena, max_struct=slots)
        srv.set_row_reuse(args.row_reuse == "on")
        return srv

    # 1. saturation: every request queued at t = 0
    srv = new_server()
    t0 = time.perf_counter()
    tickets = [submit(srv, r) for r in stream]
    srv.drain()
    wall = time.perf_counter() - t0
    sat = [srv.wait(tk) for tk in tickets]
    st = srv.stats()
    rows = srv.rows()
    srv.close()
    rate_sat = count / wall
    # 2. Poisson arrivals at 30%, 60% and 90% of the saturation rate: latency
    def poisson(fraction, seed):
        rate = fraction * rate_sat
        rng = np.random.default_rng(seed)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, count))
        srv = new_server()
        t0 = time.perf_counter()
        tickets = []
        for r, ta in zip(stream, arrivals):
            dt_wait = ta - (time.perf_counter() - t0)
            if dt_wait > 0:
                time.sleep(dt_wait)
            tickets.append(submit(srv, r))
        srv.drain()
        wall_p = time.perf_counter() - t0
        res = [srv.wait(tk) for tk in tickets]
        srv.close()
        lat = [x["t_done"] - x["t_submit"] for x in res]
        lat_sp = [x for x, r in zip(lat, stream) if r["md_steps"] == 0]
        lat_md = [x for x, r in zip(lat, stream) if r["md_steps"] > 0]
        return {"rate_fraction": fraction, "arrival_rate_per_s": rate, "wall_s": wall_p,
                "p50": _percentile_ms(lat, 50), "p99": _percentile_ms(lat, 99),
                "single_point_p50": _percentile_ms(lat_sp, 50),
                "single_point_p99": _percentile_ms(lat_sp, 99),
                "nve100_p50": _percentile_ms(lat_md, 50),
                "nve100_p99": _percentile_ms(lat_md, 99)}

    sweep = [poisson(f, 5 + k) for k, f in enumerate((0.3, 0.6, 0.9))]
    # 3. the plain path on a sample: one request at a time, host buffers in and out
    plain_pot = nepx.Potential(path, max_atoms=8192)
    step = max(1, count // max(1, args.plain_sample))
    picked = list(range(0, count, step))[:args.plain_sample]   # spread over the stream
    sample = [stream[k] for k in picked]
    t0 = time.perf_counter()
    for r in sample:
        tt = torch.as_tensor(r["type"], device="cuda")
        pp = torch.as_tensor(np.ascontiguousarray(r["pos"]), device="cuda")
        if r["md_steps"] == 0:
            pe, f, _ = plain_pot.compute(tt, r["h"], pp)
            pe.cpu(), f.cpu()
        else:
            md = nepx.MD(plain_pot, r["type"], r["mass"], r["pos"], r["vel"], r["h"])
            md.set_ensemble("nve")
            md.run(r["md_steps"], 1.0)
            md.state()
            md.close()
    torch.cuda.synchronize()
    plain_wall = time.perf_counter() - t0
    plain_work = float(sum(work[k] for k in picked))
    plain_rate = plain_work / plain_wall
    served_rate = total_atom_steps / wall
    n_atoms = [len(r["type"]) for r in stream]
    return {
        "metric": "served structures/s", "value": rate_sat, "unit": "structures/s",
        "n_gpus": 1, "higher_is_better": True,
        "dtype": "fp32 descriptors and forces, %s ANN, fp64 integration" %
                 ({"mixed": "tcgen05 FP16 (per-layer power-of-two scaling, FP32 accumulation)",
                   "mixed_bf16": "tcgen05 BF16 (FP32 accumulation)"}.get(args.precision, "fp32")),
        "data": "synthetic (seeded structures and NEP5 weights)",
        "config": {"workload": "serving_stream_%d_structs_16-8192_atoms_nep5_4type_rc5.0-4.0"
                               "_H64_20pct_nve100" % count,
                   "arena_atoms": arena, "slots": slots, "mean_atoms": float(np.mean(n_atoms)),
                   "md_fraction": float(np.mean([r["md_steps"] > 0 for r in stream]))},
        "atom_steps_per_s": served_rate,
        "saturation": {"wall_s": wall, "steps": st["steps"], "mean_resident_atoms":
                       st["mean_atoms"], "mean_resident_structs": st["mean_structs"]},
        "row_reuse": {"on": args.row_reuse == "on", "candidate_builds": rows["builds"],
                      "kept_center_steps": rows["kept"],
                      "reused_fraction": (1.0 - rows["builds"] / rows["kept"])
                      if rows["kept"] else None},
        "latency_ms": sweep[1],   # Poisson arrivals at 60% of saturation
        "latency_sweep_ms": sweep,
        "plain_fp32_one_at_a_time": {"atom_steps_per_s": plain_rate, "requests": len(sample),
                                     "wall_s": plain_wall},
        "batched_over_plain": served_rate / plain_rate,
    }


def build_system(name, seed, ncell=100):
    if name == "water":
        t, h, p = workloads.water(n_mol=8000, seed=seed)
    elif name == "carbon":
        t, h, p = workloads.diamond(a=3.567, ncell=8, jitter=0.05, seed=seed)
    elif name == "carbon8m":
        # 8,000,000 atoms (100^3 cubic cells of 8); a random 10% of the atoms
        # displaced by N(0, 0.3 A) (amorphous regions)
        t, h, p = workloads.displaced_diamond(ncell=ncell, seed=seed)
    else:
        t, h, p = workloads.fcc(a=3.615, ncell=63, vacancy=0.01, seed=seed)
    return t, h, p


def cpu_sample_system(name, seed=1):
    """The bounded sample of a workload that the CPU evaluator is timed on: the
    whole system when it is small, else a periodic block of the same lattice
    with the same vacancy / displacement statistics (the per-atom work of an
    O(N) evaluator is that of the full system).  Returns (t, h, p, what)."""
    if name == "carbon8m":
        t, h, p = workloads.displaced_diamond(ncell=20, seed=seed)
        return t, h, p, ("periodic 20x20x20-cell block (64,000 atoms) of the same displaced "
                         "diamond, every atom a center")
    if name == "copper":
        t, h, p = workloads.fcc(a=3.615, ncell=20, vacancy=0.01, seed=seed)
        return t, h, p, ("periodic 20x20x20-cell block (%d atoms) of the same FCC Cu with 1%% "
                         "vacancies, every atom a center" % len(t))
    t, h, p = build_system(name, seed)
    return t, h, p, "the full system (%d atoms)" % len(t)


def flops_per_atom(info, nr, na):
    """FP32 operations per atom of the fused descriptor/ANN/angular-force kernel.

    Counts the algorithm the kernel runs (FMA = 2): per radial edge geometry
    (~20), cutoff (~12), Chebyshev basis (4 kR) and the type-pair contraction
    (2 nR kR); per angular edge the same with kA, nA plus harmonics (~3 nlm)
    and the moment update (2 nA nlm); per center invariants, the ANN forward
    and backward (4 dim H + 12 H) and the moment derivatives (4 nA nlm); per
    angular edge of the force sweep geometry, cutoff and basis with
    derivatives (8 kA), g and g' (4 nA kA), the A/B coefficients (4 nA nlm)
    and the harmonic-gradient walk (~10 nlm).
    """
    nR, nA = info["n_max_r"] + 1, info["n_max_a"] + 1
    kR, kA = info["basis_r"] + 1, info["basis_a"] + 1
    nlm = (info["L_max"] + 1) ** 2 - 1
    dim, H = info["dim"], info["H"]
    radial = nr * (20 + 12 + 4 * kR + 2 * nR * kR)
    angular_desc = na * (20 + 12 + 4 * kA + 2 * nA * kA + 3 * nlm + 2 * nA * nlm)
    center = nA * (3 * nlm + 60) + 4 * dim * H + 12 * H + 4 * nA * nlm
    angular_force = na * (20 + 14 + 8 * kA + 4 * nA * kA + 4 * nA * nlm + 10 * nlm + 10)
    return radial + angular_desc + center + angular_force


def gather_flops_per_atom(info, nr, na):
    """FP32 operations per atom of k_gather: per radial edge geometry (~20),
    cutoff (~12), basis values and derivatives (8 kR), the two alpha dot
    products (4 kR) and the force / virial update (~30); per angular edge the
    exchange F_i += f12(i,j) - f12(j,i) and the virial (~24), plus ZBL (~60)
    for NEP-ZBL models."""
    kR = info["basis_r"] + 1
    radial = nr * (20 + 12 + 8 * kR + 4 * kR + 30)
    angular = na * (24 + (60 if info.get("zbl") else 0))
    return radial + angular


class ClockSampler:
    """nvidia-smi SM clock / throttle-reason sampling during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu_id), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for name, val in zip(names, parts[4:8]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference_rate(nep_path, sample, budget_s=8.0, max_reps=5):
    """The reference's NEP3_CPU on a bounded sample (t, h, p, what) of the
    workload on all host cores: force-call atom-steps/s, and md_step with a
    CPU velocity-Verlet update around it.  None when the reference library
    is not built."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if not oracle.ref_cpu_available():
        return None
    t, h, p, what = sample
    threads = os.cpu_count() or 1
    ref = oracle.RefCpuModel(nep_path)
    ref.compute(t, h, p, threads=threads)           # warm (thread pool, pages)
    times = []
    t_end = time.perf_counter() + budget_s
    result = None
    while len(times) < max_reps and time.perf_counter() < t_end:
        t0 = time.perf_counter()
        result = ref.compute(t, h, p, threads=threads)
        times.append(time.perf_counter() - t0)
    sec = statistics.median(times)
    n = len(t)
    line = {"value": n / sec, "unit": "atom-steps/s", "cores": threads, "kind": "reference",
            "sample": "NEP3_CPU (reference FP64 CPU evaluator) force call on %s, median of %d "
                      "calls, %d threads" % (what, len(times), threads)}
    # with a CPU velocity-Verlet loop around it: both half kicks, the drift and
    # the wrap into the box (FP64, vectorised over atoms)
    L = np.diag(np.asarray(h, dtype=np.float64).reshape(3, 3))[:, None]
    x = np.array(p, dtype=np.float64)
    v = np.zeros_like(x)
    f = np.asarray(result[1])
    inv_m = np.ones(n)
    vv = []
    for _ in range(5):
        t0 = time.perf_counter()
        v += 0.5 * 1e-3 * f * inv_m
        x += 1e-3 * v
        x -= np.floor(x / L) * L
        v += 0.5 * 1e-3 * f * inv_m
        vv.append(time.perf_counter() - t0)
    vv_s = statistics.median(vv)
    line["md_step"] = {"value": n / (sec + vv_s), "unit": "atom-steps/s",
                       "what": "force call plus a CPU velocity-Verlet update (numpy, FP64)",
                       "vv_ms": vv_s * 1e3}
    return line


def errors_vs(ref, pe, f):
    """Force RMSE / max and energy errors per atom of (pe, f) against ref."""
    pe0, f0 = ref[0], ref[1]
    n = len(pe0)
    return {"force_rmse_eV_per_A": float(np.sqrt(np.mean((f - f0) ** 2))),
            "force_max_abs_eV_per_A": float(np.abs(f - f0).max()),
            "force_rel_2norm": float(np.linalg.norm(f - f0) / np.linalg.norm(f0)),
            "energy_mae_eV_per_atom": float(np.abs(pe - pe0).mean()),
            "energy_total_eV_per_atom": float(abs(pe.sum() - pe0.sum()) / n)}


def fp64_errors(nep_path, rc_max, t, h, p, outs, clusters=9, r_core=20.0, seed=5):
    """Errors of GPU results outs = {label: (pe, f)} on the state (t, h, p)
    against the reference's FP64 NEP3_CPU.  Systems up to 100k atoms are
    evaluated whole; larger ones on `clusters` spherical cut-outs around
    random atoms (core radius r_core, shell 2 rc: the cores' energies and
    forces equal the full system's), the cores' atoms compared."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if not oracle.ref_cpu_available():
        return None
    threads = os.cpu_count() or 1
    ref = oracle.RefCpuModel(nep_path)
    n = len(t)
    if n <= 100000:
        pe0, f0, _ = ref.compute(t, h, p, threads=threads)
        idx = np.arange(n)
        what = "NEP3_CPU (reference, FP64) on the whole final MD state (%d atoms)" % n
    else:
        rng = np.random.default_rng(seed)
        pe_l, f_l, idx_l = [], [], []
        for c in rng.choice(n, clusters, replace=False):
            tc, hc, pc, core, orig = workloads.cutout(t, h, p, int(c), r_core, 2 * rc_max + 0.1)
            pe_c, f_c, _ = ref.compute(tc, hc, pc, threads=threads)
            pe_l.append(pe_c[core])
            f_l.append(f_c[:, core])
            idx_l.append(orig)
        pe0, f0, idx = np.concatenate(pe_l), np.concatenate(f_l, axis=1), np.concatenate(idx_l)
        what = ("NEP3_CPU (reference, FP64) on %d spherical cut-outs of the final MD state "
                "(core radius %.0f A, shell 2 rc): %d core atoms compared"
                % (clusters, r_core, len(idx)))
    out = {"against": what}
    for label, (pe, f) in outs.items():
        out[label] = errors_vs((pe0, f0), pe[idx], f[:, idx])
    return out


def nve_drift(precision, steps=20000, long_steps=200000, every=100, equilibrate=10000):
    """NVE energy drift of the diamond-carbon workload (8x8x8 cells, 4096
    atoms, synthetic NEP4, 300 K, dt 1 fs): least-squares slope of the total
    energy per atom against time, the reference's definition
    (tests/long_nve/long_nve_common.py nve_metrics), in eV/atom/ns.

    Two windows: 20 ps from the lattice with Maxwell-Boltzmann velocities
    (the reference's long NVE run), where kinetic energy flows into the
    lattice over the first picoseconds and velocity Verlet's O(dt^2) energy
    offset moves with it; and 200 ps after `equilibrate` steps of Berendsen
    NVT at 300 K, where what is left is the integrator's and the arithmetic's
    drift.  The total energy of a 4096-atom NVE system fluctuates by ~1e-7
    eV/atom over picoseconds (the shadow-energy offset follows the kinetic /
    potential split), so the slope of one 20 ps window scatters by about
    2e-5 eV/atom/ns whatever the precision; over 200 ps it resolves a few
    1e-6.  The long window reports its slope, the slope's standard error from
    ten block means, and the mean and spread of the slopes of its ten 20 ps
    sub-windows.  The model's neighbour-row capacities are raised to MN
    200/150: over tens of picoseconds the random-weight model densifies parts
    of the crystal, and its largest angular row (about 74) would reach the
    workload's 75."""
    import nepx
    spec = WORKLOADS["carbon"]
    tmp = tempfile.mkdtemp()
    path = workloads.write_nep(os.path.join(tmp, "nep.txt"), **dict(spec["nep"], mn=(200, 150)))
    t, h, p = build_system("carbon", seed=3)
    masses = np.full(len(t), MASSES["C"])
    v = workloads.maxwell_boltzmann(masses, 300.0, seed=4)
    pot = nepx.Potential(path, max_atoms=len(t))
    pot.set_precision(precision)

    def window(md, nsteps, blocks=0):
        try:
            rows = md.run(nsteps, 1.0, thermo_every=every)
        except nepx.NepxError as exc:   # reported in the line instead of ending the bench
            return {"error": str(exc)}
        e = (rows[:, 1] + rows[:, 2]) / len(t)
        time_ns = np.arange(1, len(e) + 1) * every * 1.0e-6
        out = {"drift_eV_per_atom_per_ns": float(np.polyfit(time_ns, e, 1)[0]),
               "max_excursion_eV_per_atom": float(np.abs(e - e[0]).max()),
               "ps": nsteps * 1.0e-3}
        if blocks:
            m = len(e) // blocks
            sub = [float(np.polyfit(time_ns[k * m:(k + 1) * m], e[k * m:(k + 1) * m], 1)[0])
                   for k in range(blocks)]
            bt = np.array([time_ns[k * m:(k + 1) * m].mean() for k in range(blocks)])
            be = np.array([e[k * m:(k + 1) * m].mean() for k in range(blocks)])
            c = np.polyfit(bt, be, 1)
            r = be - np.polyval(c, bt)
            out["slope_stderr_blocks"] = float(
                np.sqrt((r ** 2).sum() / (blocks - 2) / ((bt - bt.mean()) ** 2).sum()))
            out["sub_windows_ps"] = nsteps * 1.0e-3 / blocks
            out["sub_window_drift_mean"] = float(np.mean(sub))
            out["sub_window_drift_std"] = float(np.std(sub))
        return out

    md = nepx.MD(pot, t, masses, p, v, h)
    md.set_ensemble("nve")
    md.run(1, 1.0)
    out = window(md, steps)
    md.close()
    md = nepx.MD(pot, t, masses, p, v, h)
    md.set_ensemble("nvt_ber", T0=300.0, Tdamp=100.0)
    try:
        md.run(equilibrate, 1.0)
        md.set_ensemble("nve")
        out["equilibrated"] = window(md, long_steps, blocks=10)
    except nepx.NepxError as exc:
        out["equilibrated"] = {"error": str(exc)}
    out["equilibrated"]["nvt_ber_steps_before"] = equilibrate
    md.close()
    pot.close()
    out.update({"steps": steps, "dt_fs": 1.0, "atoms": len(t)})
    return out


def gpu_reference_rate(nep_path, t, h, p, reps=None):
    """The reference's own FP32 GPU NEP (its src/gpumd_compat kernels built for
    sm_100a, oracle/_ref) on this GPU: force calls on static positions (the
    Verlet list is built by the first call and kept), CUDA events on the
    legacy default stream the reference launches on, L2 holding the inputs."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    try:
        import torch
    except ImportError:
        return None
    if not (oracle.ref_gpu_available() and torch.cuda.is_available()):
        return None
    n = len(t)
    if reps is None:
        reps = max(5, min(50, 1200000 // n))
    d_type = torch.as_tensor(np.asarray(t, dtype=np.int32), device="cuda")
    d_pos = torch.as_tensor(np.ascontiguousarray(p, dtype=np.float64), device="cuda")
    ref = oracle.RefGpuModel(nep_path, n)
    ref.set_atoms(d_type, d_pos)
    for _ in range(3):
        ref.compute(h)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        ref.compute(h)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / reps
    del ref
    return {"value": n / (ms / 1e3), "unit": "atom-steps/s", "ms_per_call": ms,
            "kind": "reference GPU FP32 NEP (its gpumd_compat kernels, sm_100a)",
            "sample": "%d force calls on %d atoms after 3 warm-up calls, static positions"
                      % (reps, n)}


def mixed_sweep():
    """Force-call time of the FP32 and mixed-precision paths on the water
    system (24,000 atoms) for NEP models of growing descriptor and ANN size
    (two types, basis 8/8, l_max 4 2 1, the water workload's cutoffs and
    weight distribution): where the tensor-core ANN starts to pay.  Device
    time per call from nepx_profile (best of three sets of 30 calls, L2 warm)."""
    import torch
    import nepx
    t, h, p = build_system("water", seed=1)
    tt = torch.as_tensor(np.asarray(t, dtype=np.int32), device="cuda")
    pp = torch.as_tensor(np.ascontiguousarray(p), device="cuda")
    out = []
    for nmax, H in [((4, 4), 50), ((4, 4), 100), ((8, 8), 64), ((8, 8), 100), ((8, 8), 200),
                    ((12, 8), 120)]:
        spec = dict(WORKLOADS["water"]["nep"], n_max=nmax, H=H, l_max=(4, 2, 1))
        path = workloads.write_nep(os.path.join(tempfile.mkdtemp(), "nep.txt"), **spec)
        pot = nepx.Potential(path, max_atoms=len(t))
        us = {}
        for prec in ("fp32", "mixed"):
            pot.set_precision(prec)
            pot.compute(tt, h, pp, sync_check=True)
            best = min((pot.profile(tt, h, pp, reps=30) for _ in range(3)),
                       key=lambda d: d["total"])
            us[prec] = best["total"] * 1000.0
        out.append({"n_max": list(nmax), "H": H, "dim": pot.info["dim"],
                    "fp32_us": round(us["fp32"], 1), "mixed_us": round(us["mixed"], 1),
                    "mixed_over_fp32": round(us["fp32"] / us["mixed"], 3)})
        pot.close()
    return {"mixed_sweep": out, "workload": WORKLOADS["water"]["desc"]}


def headline_config(name, n, world, chunk, ncell=100):
    """The `config` of a bench line; both arms print the same dict."""
    spec = workload_spec(name, ncell)
    return {"workload": spec["desc"], "atoms_per_gpu": n, "ensemble": spec["ens"]["kind"],
            "dt_fs": spec["dt"], "parallelism": "replicas x%d" % world,
            "l2": L2_NOTE % chunk}


def run_reference_arm(args, rank):
    """The reference's own CPU implementation of the path: NEP3_CPU force call
    plus a CPU velocity-Verlet update per step, on the bounded sample of the
    workload (a periodic block of the same lattice for the large systems),
    all host threads; rank 0 only.  reference_gpu: the reference's own GPU
    kernels on the full system."""
    if rank != 0:
        return 0
    if args.workload == "serving":
        print(json.dumps({"impl": "reference", "unavailable": "the reference evaluates one "
                          "system per process: it has no batched or served path"}))
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if not oracle.ref_cpu_available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference NEP3_CPU library oracle/_ref not built"}))
        return 0
    spec = workload_spec(args.workload, args.ncell)
    chunk = max(1, min(args.chunk, args.steps))
    with tempfile.TemporaryDirectory() as tmp:
        path = workloads.write_nep(os.path.join(tmp, "nep.txt"), **spec["nep"])
        t, h, p = build_system(args.workload, seed=1, ncell=args.ncell)
        n = len(t)
        sample = cpu_sample_system(args.workload)
        ts, hs, ps, what = sample
        m = len(ts)
        syms = spec["nep"]["symbols"]
        inv_m = 1.0 / np.array([MASSES[syms[k]] for k in ts])
        L = np.diag(np.asarray(hs, dtype=np.float64).reshape(3, 3))[:, None]
        threads = os.cpu_count() or 1
        ref = oracle.RefCpuModel(path)
        x = np.array(ps, dtype=np.float64)
        v = np.zeros_like(x)
        dt = spec["dt"] / 10.18050571        # fs -> natural units (A, eV, amu)

        # one step of velocity Verlet needs one new force call; the first
        # half kick reuses the previous step's force
        _, f, _ = ref.compute(ts, hs, x, threads=threads)
        for _ in range(args.warmup):
            v += 0.5 * dt * f * inv_m
            x += dt * v
            x -= np.floor(x / L) * L
            _, f, _ = ref.compute(ts, hs, x, threads=threads)
            v += 0.5 * dt * f * inv_m
        t0 = time.perf_counter()
        for _ in range(args.steps):
            v += 0.5 * dt * f * inv_m
            x += dt * v
            x -= np.floor(x / L) * L
            _, f, _ = ref.compute(ts, hs, x, threads=threads)
            v += 0.5 * dt * f * inv_m
        sec = (time.perf_counter() - t0) / args.steps
        value = m / sec
        ref_gpu = gpu_reference_rate(path, t, h, p)
    line = {"impl": "reference", "metric": "atom-steps/s", "value": value,
            "unit": "atom-steps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * n / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp64",
            "data": "synthetic (seeded structure, velocities and NEP weights)",
            "config": headline_config(args.workload, n, args.gpus, chunk, args.ncell),
            "cpu_baseline": {"value": value, "unit": "atom-steps/s", "cores": threads,
                             "kind": "reference",
                             "sample": "per step: NEP3_CPU (reference FP64 CPU evaluator) force "
                                       "call and a velocity-Verlet update (numpy, FP64) on %s; "
                                       "ms_per_step scales the sample's time to the %d atoms "
                                       "of the config" % (what, n)},
            "e2e": {"value": value, "unit": "atom-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "reference_gpu": ref_gpu}
    print(json.dumps(line))
    return 0


class Ranks:
    """Rank plumbing of the replica runs (one independent system per GPU, no
    collective on the data path): barriers and the max / sum over ranks of a
    scalar, on the initialised process group (NCCL on GPUs, gloo on CPU).
    With no group every operation is the identity."""

    def __init__(self, dist=None, device="cpu"):
        self.dist = dist
        self.device = device

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def _reduce(self, x, op):
        if not self.dist:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x):
        return self._reduce(x, self.dist.ReduceOp.MAX if self.dist else None)

    def sum(self, x):
        return self._reduce(x, self.dist.ReduceOp.SUM if self.dist else None)


def replica_rate(units_per_rank, steps, ms_per_rank, ranks):
    """Whole-job throughput of N replicas: every rank's units over the
    slowest rank's time (max over ranks)."""
    total = ranks.sum(units_per_rank)
    ms = ranks.max(ms_per_rank)
    return total * steps / (ms / 1e3), ms

def workload_spec(name, ncell=100):
    """The workload's spec; the large carbon system at another size when
    ncell (cubic cells per edge) is not 100."""
    spec = WORKLOADS[name]
    if name == "carbon8m" and ncell != 100:
        spec = dict(spec, desc=spec["desc"].replace(
            "100x100x100cells_8000000atoms", "%dx%dx%dcells_%datoms" % (ncell, ncell, ncell,
                                                                       8 * ncell ** 3)))
    return spec


def md_system(name, rank, ncell=100):
    """Potential file, structure, masses and 300 K velocities of a workload."""
    spec = workload_spec(name, ncell)
    path = workloads.write_nep(os.path.join(tempfile.mkdtemp(), "nep.txt"), **spec["nep"])
    t, h, p = build_system(name, seed=1 + rank, ncell=ncell)
    syms = spec["nep"]["symbols"]
    masses = np.array([MASSES[x] for x in syms])[t]
    v = workloads.maxwell_boltzmann(masses, spec["T"], seed=7 + rank)
    return dict(name=name, spec=spec, path=path, t=t, h=h, p=p, masses=masses, v=v)


def new_md(pot, sysd, rank, warmup):
    import nepx
    spec = sysd["spec"]
    md = nepx.MD(pot, sysd["t"], sysd["masses"], sysd["p"], sysd["v"], sysd["h"])
    ens = dict(spec["ens"])
    kind = ens.pop("kind")
    md.set_ensemble(kind, seed=12345678 + rank, **ens)
    md.run(warmup, spec["dt"])
    return md


def timed_md(pot, sysd, args, rank, ranks, flush, clocks=None):
    """K MD steps in chunks, each after an L2 flush, timed by CUDA events on
    the MD stream: (device ms, final state, clocks, number of chunks)."""
    import torch
    dt = sysd["spec"]["dt"]
    md = new_md(pot, sysd, rank, args.warmup)
    _, _, _, _, stream_ptr = md.device_state()
    stream = torch.cuda.ExternalStream(stream_ptr)
    K, chunk = args.steps, max(1, min(args.chunk, args.steps))
    chunks = [chunk] * (K // chunk) + ([K % chunk] if K % chunk else [])
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in chunks]
    ranks.barrier()
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
        time.sleep(0.2)
    for c, steps in enumerate(chunks):
        with torch.cuda.stream(stream):
            flush.fill_(c & 0xFF)
        ev[c][0].record(stream)
        md.run_async(steps, dt)
        ev[c][1].record(stream)
    md.sync()
    torch.cuda.synchronize()
    clock_info = clocks.stop() if clocks else None
    ranks.barrier()
    dev_ms = sum(a.elapsed_time(b) for a, b in ev)
    st = md.state()
    md.close()
    return dev_ms, st, clock_info, len(chunks)


def force_call_profile(pot, sysd, st, reps):
    """Per-stage device time (nepx_profile) and the outputs (pe, f as numpy)
    of one force call on the state st, at the handle's current precision."""
    import torch
    tt = torch.as_tensor(np.asarray(sysd["t"], dtype=np.int32), device="cuda")
    pp = torch.as_tensor(np.ascontiguousarray(st["pos"]), device="cuda")
    prof = pot.profile(tt, st["h"], pp, reps=reps)
    pe, f, _ = pot.compute(tt, st["h"], pp, sync_check=True)
    out = (pe.cpu().numpy(), f.cpu().numpy())
    del tt, pp, pe, f
    return prof, out


def mean_neighbors(pot, n):
    """Mean radial and angular row lengths of the last force call (the first
    262,144 atoms of a larger system)."""
    m = min(n, 262144)
    return float(pot.neighbor_counts(0, m).mean()), float(pot.neighbor_counts(1, m).mean())


# ncu on the tensor-core build of the descriptor kernel (one launch, 1,000,000
# atoms of the large-carbon system, --set full): sm__pipe_tensor_cycles_active
# and sm__pipe_tc_cycles_active, percent of the launch's cycles
TENSOR_PIPE_ACTIVE_PCT = {"tensor": 0.63, "tc": 2.27}


def ann_tensor_fraction(sysd, atom_steps_per_s):
    """The ANN's algorithmic work on the tensor cores: 4 dim H FLOP per atom
    (forward and backward contraction, FMA = 2) at the mixed MD's rate, as a
    fraction of the measured dense bf16 peak (the FP16 MMAs run at the same
    rate), with the tensor-pipe activity ncu measured."""
    nep = sysd["spec"]["nep"]
    n_r, n_a = nep["n_max"][0] + 1, nep["n_max"][1] + 1
    l3 = nep["l_max"]
    dim = n_r + n_a * (l3[0] + (1 if l3[1] else 0) + (1 if l3[2] else 0))
    flops = 4 * dim * nep["H"]
    peak = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peak = json.load(fh).get("bf16_tflops")
    except (OSError, ValueError):
        pass
    achieved = atom_steps_per_s * flops / 1e12
    return {"flops_per_atom": flops, "dim": dim, "H": nep["H"], "achieved_tflops": achieved,
            "peak_tflops": peak, "peak_source": "MEASURED_PEAKS.json bf16_tflops (measured)",
            "frac": achieved / peak if peak else None,
            "pipe_active_pct_ncu": TENSOR_PIPE_ACTIVE_PCT}


def force_kernels(pot):
    """The force kernels of a Verlet-row force call with the handle's launch
    choices: the angular partial forces come from the descriptor kernel
    itself or from k_angular_f12."""
    fused = pot.tuning()[0]["fused_f12"] == 1
    return ["k_filter_radial", "k_nep_fused"] + ([] if fused else ["k_angular_f12"]) + ["k_gather"]


def roofline_of(pot, name, n, prof):
    """The force kernels against the FP32 FMA peak (stage times of prof)."""
    mean_r, mean_a = mean_neighbors(pot, n)
    info = dict(pot.info)
    fpa = flops_per_atom(info, mean_r, mean_a)
    gfa = gather_flops_per_atom(info, mean_r, mean_a)
    ms = prof["descriptor"] + prof["gather"]
    achieved = (fpa + gfa) * n / (ms * 1e-3) / 1e12
    peak = FP32_LANES * 2 * SM_MAX_MHZ * 1e6 / 1e12
    per_atom = TRAFFIC_PER_ATOM.get((name, tuple(force_kernels(pot))))
    return {"bound": "fp32",
            "kernel": " + ".join(force_kernels(pot)) + " (force stage)",
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "traffic": per_atom * n if per_atom else None,
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the force "
                              "kernels, one launch each, per atom of the captured system "
                              "times this system's atoms",
            "peak_source": "B200 FP32 FMA peak: 148 SMs x 128 lanes x 2 FLOP x 1965 MHz "
                           "(not in MEASURED_PEAKS.json, which holds HBM and bf16 only); "
                           "fraction of that nominal peak",
            "timing": "CUDA events around the stages of nepx_profile (force calls on the final "
                      "MD state, L2 holding what fits)",
            "ms_per_launch": ms, "flops_per_atom": fpa + gfa,
            "flops_per_atom_descriptor_stage": fpa, "flops_per_atom_gather": gfa,
            "mean_radial_neighbors": mean_r, "mean_angular_neighbors": mean_a}


def profile_reps(n):
    return max(5, min(50, 1200000 // n))


def other_workload(name, args, rank, ranks, flush):
    """MD rate (FP32 and mixed), force call and FP64 errors of a secondary
    workload, for the extra keys of the headline line."""
    import nepx
    sysd = md_system(name, rank)
    n = len(sysd["t"])
    pot = nepx.Potential(sysd["path"], max_atoms=n)
    dev_ms, st, _, _ = timed_md(pot, sysd, args, rank, ranks, flush)
    prof, out32 = force_call_profile(pot, sysd, st, profile_reps(n))
    pot.set_precision("mixed")
    dev_ms_m, _, _, _ = timed_md(pot, sysd, args, rank, ranks, flush)
    prof_m, outm = force_call_profile(pot, sysd, st, profile_reps(n))
    pot.set_precision("fp32")
    roof = roofline_of(pot, name, n, prof)
    pot.close()
    value = n * args.steps / (dev_ms * 1e-3)
    line = {"workload": sysd["spec"]["desc"], "atoms": n, "ensemble": sysd["spec"]["ens"]["kind"],
            "value": value, "unit": "atom-steps/s", "ms_per_step": dev_ms / args.steps,
            "steps": args.steps,
            "mixed_precision": {"value": n * args.steps / (dev_ms_m * 1e-3),
                                "over_fp32": dev_ms / dev_ms_m, "stage_ms": prof_m,
                                "ann_tensor": ann_tensor_fraction(
                                    sysd, n * args.steps / (dev_ms_m * 1e-3))},
            "force_call": {"ms": prof["total"], "stage_ms": prof,
                           "value": n / (prof["total"] * 1e-3)},
            "roofline": roof}
    if not args.no_cpu_baseline:
        rc_max = max(sysd["spec"]["nep"]["rc"])
        line["err_vs_fp64"] = fp64_errors(sysd["path"], rc_max, sysd["t"], st["h"], st["pos"],
                                          {"fp32": out32, "mixed": outm})
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="carbon8m", choices=sorted(WORKLOADS) + ["serving"])
    ap.add_argument("--requests", type=int, default=20000)
    ap.add_argument("--arena", type=int, default=262144)
    ap.add_argument("--plain-sample", type=int, default=200)
    ap.add_argument("--chunk", type=int, default=10)
    ap.add_argument("--ncell", type=int, default=100,
                    help="cubic cells per edge of the large carbon workload (8 atoms each)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mixed-sweep", action="store_true",
                    help="print FP32 vs mixed force-call times over NEP model sizes and exit")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the other workloads, the NVE drift and the serving sample")
    ap.add_argument("--serving-sample", type=int, default=5000)
    ap.add_argument("--row-reuse", default="on", choices=["on", "off"],
                    help="serving: MD segments keep Verlet candidates between steps")
    ap.add_argument("--precision", default="mixed", choices=["fp32", "mixed", "mixed_bf16"],
                    help="ANN precision of the serving workload")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank)
    if args.workload == "serving":
        if rank == 0:
            print(json.dumps(run_serving(args)))
        return 0
    if args.mixed_sweep:
        if rank == 0:
            print(json.dumps(mixed_sweep()))
        return 0

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    ranks = Ranks(dist, "cuda")
    import nepx

    sysd = md_system(args.workload, rank, args.ncell)
    spec = sysd["spec"]
    t, h, p = sysd["t"], sysd["h"], sysd["p"]
    n = len(t)
    dt = spec["dt"]
    kind = spec["ens"]["kind"]
    K = args.steps
    chunk = max(1, min(args.chunk, args.steps))
    pot = nepx.Potential(sysd["path"], max_atoms=n)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    props = torch.cuda.get_device_properties(local)
    gpu_id = getattr(props, "uuid", None)
    gpu_id = ("GPU-" + str(gpu_id)) if gpu_id is not None else local
    clocks = ClockSampler(gpu_id)

    # 1. the headline: FP32 MD, device time
    dev_ms, st, clock_info, nchunks = timed_md(pot, sysd, args, rank, ranks, flush, clocks)
    value, dev_ms = replica_rate(n, K, dev_ms, ranks)
    # k_vv1 (with the skin check), k_neighbor_rebuild (returns at once unless
    # a rebuild is due), the force kernels, k_vv2_thermo, k_ensemble, k_scale;
    # NHC adds two
    kernels_per_step = 5 + len(force_kernels(pot)) + (2 if kind == "nvt_nhc" else 0)
    # per call (chunk): k_mark_call before the step graphs and k_publish after
    # them; the L2-flush fills are torch's, not counted
    launches = K * kernels_per_step + 2 * nchunks

    # 2. end to end through the public API: one nepx_md_run per step over the
    # same steps from the same initial state
    md = new_md(pot, sysd, rank, args.warmup)
    rows = None
    ranks.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(K):
        rows = md.run(1, dt, thermo_every=1)
    e2e_value, _ = replica_rate(n, K, (time.perf_counter() - t0) * 1e3, ranks)
    e2e = {"value": e2e_value, "unit": "atom-steps/s",
           "h2d_bytes_per_step": 8 * 8 if kind != "nve" else 0,   # stochastic draws
           # thermo row, status word, box, neighbour state
           "d2h_bytes_per_step": 20 * 8 + 4 + 232 + 128,
           "api": "nepx_md_run(steps=1, thermo_every=1) per step, the timed run's steps"}
    md.close()

    # 3. the same MD with the ANN on the tensor cores
    pot.set_precision("mixed")
    dev_ms_m, _, _, _ = timed_md(pot, sysd, args, rank, ranks, flush)
    value_mixed, dev_ms_m = replica_rate(n, K, dev_ms_m, ranks)
    reps = profile_reps(n)
    prof_mixed, out_mixed = force_call_profile(pot, sysd, st, reps)
    pot.set_precision("fp32")
    prof, out_fp32 = force_call_profile(pot, sysd, st, reps)
    roofline = roofline_of(pot, args.workload, n, prof)
    mixed = {"value": value_mixed, "unit": "atom-steps/s", "ms_per_step": dev_ms_m / K,
             "over_fp32": value_mixed / value,
             "what": "the same MD with the ANN's two contractions as tcgen05 MMAs inside the "
                     "descriptor kernel: FP16 operands with per-layer power-of-two scaling, FP32 "
                     "accumulation in TMEM; descriptors and forces FP32",
             "stage_ms": prof_mixed,
             "ann_tensor": ann_tensor_fraction(sysd, value_mixed)}
    pot.close()
    del flush
    torch.cuda.empty_cache()

    line = None
    if rank == 0:
        cpu = err = None
        if world == 1 and not args.no_cpu_baseline:
            # the reference FP64 CPU evaluator: timed on a bounded sample, and
            # the FP64 values the GPU results of the final state are checked against
            cpu = cpu_reference_rate(sysd["path"], cpu_sample_system(args.workload))
            err = fp64_errors(sysd["path"], max(spec["nep"]["rc"]), t, st["h"], st["pos"],
                              {"fp32": out_fp32, "mixed": out_mixed})
        others = drift = serving = None
        if not args.no_extras:
            flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
            others = {w: other_workload(w, args, rank, Ranks(None), flush)
                      for w in ("water", "copper") if w != args.workload}
            del flush
            drift = {"fp32": nve_drift("fp32"), "mixed": nve_drift("mixed")}
            if args.serving_sample > 0:
                sargs = argparse.Namespace(requests=args.serving_sample, arena=args.arena,
                                           plain_sample=max(20, args.serving_sample // 20),
                                           precision="mixed", row_reuse=args.row_reuse)
                sv = run_serving(sargs)
                serving = {k: sv[k] for k in ("value", "unit", "atom_steps_per_s", "latency_ms",
                                              "latency_sweep_ms", "plain_fp32_one_at_a_time",
                                              "batched_over_plain", "config", "saturation",
                                              "row_reuse")}
        T_last = float(rows[-1, 0]) if rows is not None else None
        line = {"metric": "atom-steps/s", "value": value, "unit": "atom-steps/s",
                "n_gpus": world, "steps": K, "warmup": args.warmup,
                "ms_per_step": dev_ms / K, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "fp32 (descriptors, ANN, forces) + fp64 "
                                              "(integration, thermo reductions)",
                "data": "synthetic (seeded structure, velocities and NEP weights)",
                "config": headline_config(args.workload, n, world, chunk, args.ncell),
                "final_temperature_K": T_last,
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "force_call": {"value": n / (prof["total"] * 1e-3), "unit": "atom-steps/s",
                               "ms": prof["total"], "stage_ms": prof,
                               "what": "nepx_compute on the final state, static positions "
                                       "(neighbour update + descriptor + gather)"},
                "mixed_precision": mixed, "err_vs_fp64": err, "other_workloads": others,
                "nve_drift": drift, "serving": serving,
                "gpu_launches": launches, "clocks": clock_info}
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
