"""Seeded synthetic inputs: NEP potential files and periodic structures.

Shared by the tests and bench.py.  Nothing here reads the reference tree; the
shapes, sizes and value distributions are those of the benchmark configs:

  * NEP files with weights N(0, std^2) in the GPUMD nep.txt format that both
    the reference GPU loader (nep.cu:135-415) and its CPU evaluator
    (nep_cpu.cpp:1957-2250) accept: a 5-token cutoff line and a 4-token
    l_max line;
  * diamond carbon, FCC copper with vacancies, liquid water boxes at a given
    density, random-packed multi-species boxes, and Maxwell-Boltzmann
    velocities.
"""
import math
import os

import numpy as np

MASS = {"H": 1.008, "C": 12.011, "N": 14.007, "O": 15.999, "Cu": 63.546, "Si": 28.085,
        "Ba": 137.327, "Ti": 47.867}
K_B = 8.617343e-5


def write_nep(path, version=4, symbols=("C",), zbl=None, rc=(4.2, 3.7), mn=(100, 60),
              n_max=(4, 4), basis=(8, 8), l_max=(4, 2, 1), H=30, seed=0, std=0.1,
              q_scaler=1.0):
    """Write a synthetic NEP file; returns its path.

    rc: (rc_radial, rc_angular), or one such pair per type (typewise cutoffs).
    zbl: None, (rc_inner, rc_outer), (rc_inner, rc_outer, factor) or
    "flexible" (the "zbl 0 0" form: per type pair rc_inner, rc_outer and four
    screening pairs (a_k, b_k) after the descriptor scales, drawn near the
    universal ZBL values).
    """
    T = len(symbols)
    nR, nA = n_max[0] + 1, n_max[1] + 1
    kR, kA = basis[0] + 1, basis[1] + 1
    # l_max: (L, has_q_222, has_q_1111[, has_q_112, has_q_123, has_q_233, has_q_134])
    num_L = l_max[0] + sum(1 for flag in l_max[1:] if flag)
    dim = nR + nA * num_L
    if version == 4:
        num_ann = (dim + 2) * H * T + 1
    else:
        num_ann = ((dim + 2) * H + 1) * T + 1
    num_desc = T * T * (nR * kR + nA * kA)
    rng = np.random.default_rng(seed)
    params = rng.normal(0.0, std, num_ann + num_desc)
    tag = "nep%d%s" % (version, "_zbl" if zbl else "")
    lines = ["%s %d %s" % (tag, T, " ".join(symbols))]
    if zbl == "flexible":
        lines.append("zbl 0 0")
    elif zbl:
        lines.append("zbl " + " ".join("%g" % v for v in zbl))
    if np.ndim(rc) == 2:   # per-type cutoffs: (rc_radial, rc_angular) of each type
        lines.append("cutoff " + " ".join("%g %g" % tuple(c) for c in rc) +
                     " %d %d" % (mn[0], mn[1]))
    else:
        lines.append("cutoff %g %g %d %d" % (rc[0], rc[1], mn[0], mn[1]))
    lines.append("n_max %d %d" % n_max)
    lines.append("basis_size %d %d" % basis)
    lines.append("l_max " + " ".join("%d" % v for v in l_max))
    lines.append("ANN %d 0" % H)
    lines += ["%.8e" % v for v in params]
    qs = np.full(dim, q_scaler) if np.isscalar(q_scaler) else np.asarray(q_scaler)
    lines += ["%.8e" % v for v in qs]
    if zbl == "flexible":
        universal = [0.18175, 3.1998, 0.50986, 0.94229, 0.28022, 0.4029, 0.02817, 0.20162]
        for _ in range(T * (T + 1) // 2):
            pair = [rng.uniform(0.8, 1.2), rng.uniform(1.8, 2.2)]
            pair += [c * rng.uniform(0.9, 1.1) for c in universal]
            lines += ["%.8e" % v for v in pair]
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path


# Synthetic models of the benchmark workloads (write_nep keyword arguments).
# q_scaler 0.02 keeps the random-weight landscape gentle, so the systems keep
# their density and neighbour counts through the runs.
NEP_SPECS = {
    # liquid water, O/H
    "water": dict(version=4, symbols=("O", "H"), rc=(6.0, 4.0), mn=(250, 100), n_max=(4, 4),
                  basis=(8, 8), l_max=(4, 2, 0), H=50, seed=2024, std=0.1, q_scaler=0.02),
    # diamond / amorphous carbon (4,096 and 8,000,000 atoms)
    "carbon": dict(version=4, symbols=("C",), rc=(4.2, 3.7), mn=(100, 60), n_max=(4, 4),
                   basis=(8, 8), l_max=(4, 2, 1), H=30, seed=2025, std=0.1, q_scaler=0.02),
    # FCC copper with the universal ZBL (inner 1.0 A, outer 2.0 A)
    "copper": dict(version=4, symbols=("Cu",), zbl=(1.0, 2.0), rc=(5.0, 4.0), mn=(100, 60),
                   n_max=(4, 4), basis=(8, 8), l_max=(4, 2, 1), H=40, seed=2026, std=0.1,
                   q_scaler=0.02),
    # the serving stream's shared four-type NEP5 (C, H, O, Cu)
    "serving": dict(version=5, symbols=("C", "H", "O", "Cu"), rc=(5.0, 4.0), mn=(160, 80),
                    n_max=(4, 4), basis=(8, 8), l_max=(4, 2, 1), H=64, seed=2027, std=0.1,
                    q_scaler=0.02),
}


def _cubic_h(L):
    return np.array([L, 0, 0, 0, L, 0, 0, 0, L], dtype=np.float64)


def diamond(a=3.567, ncell=8, jitter=0.05, seed=0):
    """Diamond supercell: (types, h, pos (3, n))."""
    base = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0],
                     [.25, .25, .25], [.25, .75, .75], [.75, .25, .75], [.75, .75, .25]])
    g = np.stack(np.meshgrid(*[np.arange(ncell)] * 3, indexing="ij"), -1).reshape(-1, 3)
    frac = (g[:, None, :] + base[None, :, :]).reshape(-1, 3) / ncell
    L = a * ncell
    rng = np.random.default_rng(seed)
    pos = frac * L + rng.normal(0.0, jitter, frac.shape)
    return np.zeros(len(pos), dtype=np.int32), _cubic_h(L), np.ascontiguousarray(pos.T % L)


def displaced_diamond(ncell=100, fraction=0.10, sigma=0.3, seed=1):
    """Diamond supercell (a = 3.567 A, jitter N(0, 0.05 A)) with a random
    `fraction` of the atoms displaced by N(0, sigma) (amorphous regions).
    ncell 100 gives the 8,000,000-atom large-carbon workload."""
    t, h, p = diamond(a=3.567, ncell=ncell, jitter=0.05, seed=seed)
    rng = np.random.default_rng(seed + 100)
    pick = rng.random(len(t)) < fraction
    L = h[0]
    p[:, pick] = (p[:, pick] + rng.normal(0.0, sigma, (3, int(pick.sum())))) % L
    return t, h, p


def cutout(t, h, p, center, r_core, r_shell):
    """Spherical cluster around atom `center` of an orthogonal periodic box.

    Keeps every atom within r_core + r_shell (minimum image) and places the
    cluster in a cubic box wide enough that its periodic images are more than
    r_shell / 2 apart.  With r_shell >= 2 rc the energy, force and virial of
    every atom within r_core are those of the full system (its descriptors
    and its neighbours' descriptors see the same atoms).  Returns (types, h,
    pos (3, m), core index into the cluster, original index of the core)."""
    L = np.diag(np.asarray(h, dtype=np.float64).reshape(3, 3))
    d = p - p[:, center][:, None]
    d -= np.round(d / L[:, None]) * L[:, None]
    r2 = (d * d).sum(axis=0)
    keep = np.nonzero(r2 < (r_core + r_shell) ** 2)[0]
    side = 2.0 * (r_core + r_shell) + r_shell / 2.0 + 1.0
    pos = np.ascontiguousarray(d[:, keep] + side / 2.0)
    core = np.nonzero(r2[keep] < r_core ** 2)[0]
    return (np.ascontiguousarray(t[keep]), _cubic_h(side), pos, core, keep[core])


def fcc(a=3.615, ncell=8, vacancy=0.0, jitter=0.0, seed=0):
    base = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]])
    g = np.stack(np.meshgrid(*[np.arange(ncell)] * 3, indexing="ij"), -1).reshape(-1, 3)
    frac = (g[:, None, :] + base[None, :, :]).reshape(-1, 3) / ncell
    rng = np.random.default_rng(seed)
    if vacancy > 0:
        keep = rng.random(len(frac)) >= vacancy
        frac = frac[keep]
    L = a * ncell
    pos = frac * L
    if jitter:
        pos = pos + rng.normal(0.0, jitter, pos.shape)
    return np.zeros(len(pos), dtype=np.int32), _cubic_h(L), np.ascontiguousarray(pos.T % L)


def water(n_mol=8000, density=1.0, seed=0, roh=0.96, angle=104.5):
    """Liquid-water box (types O=0, H=1) at density g/cm^3, random orientations.

    Molecules sit on a jittered cubic lattice so no two oxygens overlap.
    """
    amu_per_A3 = density * 0.60221408
    L = (n_mol * 18.015 / amu_per_A3) ** (1.0 / 3.0)
    m = int(math.ceil(n_mol ** (1.0 / 3.0)))
    rng = np.random.default_rng(seed)
    sites = np.stack(np.meshgrid(*[np.arange(m)] * 3, indexing="ij"), -1).reshape(-1, 3)
    sites = sites[rng.permutation(len(sites))[:n_mol]]
    spacing = L / m
    O = (sites + 0.5) * spacing + rng.uniform(-0.15, 0.15, (n_mol, 3)) * spacing
    th = math.radians(angle)
    local = np.array([[roh, 0, 0], [roh * math.cos(th), roh * math.sin(th), 0]])
    # random rotations from normalised quaternions
    q = rng.normal(size=(n_mol, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1)], 1)
    Hs = O[:, None, :] + np.einsum("mij,kj->mki", R, local)
    pos = np.concatenate([O[:, None, :], Hs], 1).reshape(-1, 3) % L
    types = np.tile(np.array([0, 1, 1], dtype=np.int32), n_mol)
    return types, _cubic_h(L), np.ascontiguousarray(pos.T)


def random_packed(n, num_types, density=0.08, min_dist=0.9, seed=0):
    """Random-packed box at `density` atoms/A^3 with a soft minimum distance."""
    L = (n / density) ** (1.0 / 3.0)
    rng = np.random.default_rng(seed)
    m = int(math.ceil(n ** (1.0 / 3.0)))
    sites = np.stack(np.meshgrid(*[np.arange(m)] * 3, indexing="ij"), -1).reshape(-1, 3)
    sites = sites[rng.permutation(len(sites))[:n]]
    sp = L / m
    pos = (sites + 0.5) * sp + rng.uniform(-0.25, 0.25, (n, 3)) * max(sp - min_dist, 0.0)
    types = rng.integers(0, num_types, n).astype(np.int32)
    return types, _cubic_h(L), np.ascontiguousarray((pos % L).T)


def maxwell_boltzmann(masses, T, seed=0):
    """Velocities (3, n) in A/fs with zero total momentum, scaled to T exactly."""
    rng = np.random.default_rng(seed)
    masses = np.asarray(masses, dtype=np.float64)
    # natural units: v in A / (natural time); 1 natural time = 10.18051 fs
    sigma = np.sqrt(K_B * T / masses)
    v = rng.normal(size=(3, len(masses))) * sigma
    p = (v * masses).sum(axis=1) / masses.sum()
    v -= p[:, None]
    ek = 0.5 * (masses * (v * v).sum(axis=0)).sum()
    v *= math.sqrt(1.5 * len(masses) * K_B * T / ek)
    return v / 10.18051


DIAMOND_BASE = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0],
                         [.25, .25, .25], [.25, .75, .75], [.75, .25, .75], [.75, .75, .25]])
FCC_BASE = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]])


def crystal(base, a, dims, jitter=0.0, seed=0):
    """Orthorhombic supercell dims = (nx, ny, nz) of a cubic cell with `base` sites."""
    dims = np.asarray(dims)
    g = np.stack(np.meshgrid(*[np.arange(d) for d in dims], indexing="ij"), -1).reshape(-1, 3)
    frac = (g[:, None, :] + base[None, :, :]).reshape(-1, 3)
    L = a * dims
    rng = np.random.default_rng(seed)
    pos = frac * a + rng.normal(0.0, jitter, frac.shape)
    h = np.diag(L.astype(np.float64)).reshape(-1)
    return np.zeros(len(pos), dtype=np.int32), h, np.ascontiguousarray((pos % L).T)


def _near_cubic_dims(n_atoms, per_cell):
    a = max(1, int(round((n_atoms / per_cell) ** (1.0 / 3.0))))
    c = max(1, int(round(n_atoms / (per_cell * a * a))))
    return (a, a, c)


def serving_stream(count, seed=0, md_fraction=0.2, md_steps=100, lo=16, hi=8192):
    """Independent structures of log-uniform size lo..hi atoms: jittered
    (sigma 0.1 A) diamond C and FCC Cu supercells and random-packed C/H/O/Cu
    at 0.08 atoms/A^3 (types 0..3 = C, H, O, Cu).  A fraction md_fraction of
    the requests are NVE segments of md_steps steps at 300 K.  Returns a list
    of dicts (type, h, pos, md_steps, mass, vel)."""
    rng = np.random.default_rng(seed)
    masses = np.array([12.011, 1.008, 15.999, 63.546])
    out = []
    for k in range(count):
        n = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        kind = rng.integers(0, 3)
        if kind == 0:
            t, h, p = crystal(DIAMOND_BASE, 3.567, _near_cubic_dims(n, 8), 0.1, seed + k)
        elif kind == 1:
            t, h, p = crystal(FCC_BASE, 3.615, _near_cubic_dims(n, 4), 0.1, seed + k)
            t = np.full(len(t), 3, dtype=np.int32)
        else:
            t, h, p = random_packed(n, 4, density=0.08, seed=seed + k)
        req = {"type": t, "h": h, "pos": p, "md_steps": 0, "mass": None, "vel": None}
        if rng.random() < md_fraction:
            m = masses[t]
            req.update(md_steps=md_steps, mass=m, vel=maxwell_boltzmann(m, 300.0, seed + k))
        out.append(req)
    return out
