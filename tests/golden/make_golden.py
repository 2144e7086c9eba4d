#!/usr/bin/env python3
"""Regenerate the committed golden fixtures from the DMG-MD reference tree.

Run in a checkout that has the reference available (--reference, else
$DMGMD_REFERENCE, else a `reference` directory beside this repository):

    python tests/golden/make_golden.py [--reference PATH]

It reads, as data only:
  * tests/baseline/goldens/*  -- GPUMD 5.9.1 FP32 outputs (per-atom force,
    energy, virial; NVE trajectory) of the reference's golden suite,
  * tests/baseline/inputs/*   -- the matching model.xyz / run.in inputs and
    the three NEP potential files,
  * the programs' output files (thermo.out, dump_xyz, restart.xyz and the
    neighbor.out occupancy records),
  * tests/thermostats/fixtures/{svr,nhc}.json -- bit-level thermostat KATs,
and writes tests/golden/baseline_goldens.json, tests/golden/potentials/*.txt
and tests/golden/thermostats/*.json.  The tests never read the reference
tree at run time.
"""
import argparse
import json
import os
import re
import shutil

HERE = os.path.dirname(os.path.abspath(__file__))

STATIC_CASES = {
    # case: (golden xyz, potential, force path the reference takes)
    "single_small_static": ("single_small_static/main/initial.xyz", "nep_C.txt", "small-box"),
    "single_large_nve": ("single_large_nve/main/initial.xyz", "nep_C.txt", "large-box"),
    "multi_nvt_restart": ("multi_nvt_restart/initial/initial.xyz", "nep_water.txt", "large-box"),
    "nep_zbl_boundary": ("nep_zbl_boundary/main/initial.xyz", "nep_BaTiO3_zbl.txt", "large-box"),
}


def parse_extxyz(text):
    """Return a list of frames {header: dict, columns: {name: rows}}."""
    lines = text.splitlines()
    frames = []
    k = 0
    while k < len(lines):
        if not lines[k].strip():
            k += 1
            continue
        n = int(lines[k].split()[0])
        header = lines[k + 1]
        kv = dict(re.findall(r'(\w+)=("[^"]*"|\S+)', header))
        kv = {key: val.strip('"') for key, val in kv.items()}
        props = kv["Properties"].split(":")
        cols = []
        for p in range(0, len(props), 3):
            cols.append((props[p], props[p + 1], int(props[p + 2])))
        rows = [lines[k + 2 + i].split() for i in range(n)]
        data = {}
        c = 0
        for name, kind, width in cols:
            vals = [r[c:c + width] for r in rows]
            if kind == "S":
                data[name] = [v[0] for v in vals]
            elif kind == "I":
                data[name] = [[int(x) for x in v] for v in vals]
            else:
                data[name] = [[float(x) for x in v] for v in vals]
            c += width
        frames.append({"header": kv, "data": data, "n": n})
        k += 2 + n
    return frames


def lattice_to_h(lattice):
    """extxyz Lattice="ax ay az bx by bz cx cy cz" -> row-major h with columns a, b, c."""
    a = [float(x) for x in lattice.split()]
    ax, ay, az, bx, by, bz, cx, cy, cz = a
    return [ax, bx, cx, ay, by, cy, az, bz, cz]


def species_types(potential_path):
    with open(potential_path) as f:
        head = f.readline().split()
    return head[2:2 + int(head[1])]


def frame_record(frame, symbols):
    d = frame["data"]
    pbc = [1 if t == "T" else 0 for t in frame["header"]["pbc"].split()]
    rec = {
        "n": frame["n"],
        "h": lattice_to_h(frame["header"]["Lattice"]),
        "pbc": pbc,
        "species": d["species"],
        "type": [symbols.index(s) for s in d["species"]],
        "pos": d["pos"],
        "time_fs": float(frame["header"].get("Time", 0.0)),
    }
    if "forces" in d:
        rec["force"] = d["forces"]
    if "energy_atom" in d:
        rec["energy_atom"] = [v[0] for v in d["energy_atom"]]
    if "virial" in d:
        rec["virial_rowmajor"] = d["virial"]
    if "vel" in d:
        rec["vel"] = d["vel"]
    if "energy" in frame["header"]:
        rec["energy_total"] = float(frame["header"]["energy"])
    return rec


def main():
    ap = argparse.ArgumentParser()
    default_ref = os.environ.get("DMGMD_REFERENCE") or os.path.join(
        os.path.dirname(os.path.dirname(os.path.dirname(HERE))), "reference")
    ap.add_argument("--reference", default=default_ref)
    args = ap.parse_args()
    base = os.path.join(args.reference, "tests", "baseline")
    out = {"source": "DMG-MD tests/baseline (GPUMD 5.9.1 goldens, FP32 on NVIDIA L20)",
           "tolerances": json.load(open(os.path.join(base, "manifest.json")))["tolerances"],
           "static": {}, "trajectories": {}}
    os.makedirs(os.path.join(HERE, "potentials"), exist_ok=True)
    for pot in ("nep_C.txt", "nep_water.txt", "nep_BaTiO3_zbl.txt"):
        shutil.copyfile(os.path.join(base, "inputs", "potentials", pot),
                        os.path.join(HERE, "potentials", pot))
    for case, (xyz, pot, path) in STATIC_CASES.items():
        symbols = species_types(os.path.join(base, "inputs", "potentials", pot))
        frames = parse_extxyz(open(os.path.join(base, "goldens", xyz)).read())
        rec = frame_record(frames[0], symbols)
        rec["potential"] = pot
        rec["reference_force_path"] = path
        out["static"][case] = rec
    # NVE trajectory of single_large_nve: model.xyz input + dumped frames
    symbols = species_types(os.path.join(base, "inputs", "potentials", "nep_C.txt"))
    model = parse_extxyz(open(os.path.join(base, "inputs", "single_large_nve", "model.xyz")).read())[0]
    traj = parse_extxyz(open(os.path.join(base, "goldens", "single_large_nve", "main",
                                          "trajectory.xyz")).read())
    out["trajectories"]["single_large_nve"] = {
        "potential": "nep_C.txt",
        "run_in": open(os.path.join(base, "inputs", "single_large_nve", "run.in")).read(),
        "model": frame_record(model, symbols),
        "frames": [frame_record(f, symbols) for f in traj],
        "thermo_out": open(os.path.join(base, "goldens", "single_large_nve", "main",
                                        "thermo.out")).read(),
    }
    # whole programs: run.in / model.xyz of every stage and the golden output
    # files, for the end-to-end driver tests (nepx-md)
    manifest = json.load(open(os.path.join(base, "manifest.json")))
    out["programs"] = {}
    for case, spec in manifest["cases"].items():
        pot = os.path.basename(spec["potential"])
        stages = []
        for st in spec["stages"]:
            rec = {"name": st["name"],
                   "run_in": open(os.path.join(base, st["run"])).read(),
                   "model_xyz": open(os.path.join(base, st["model"])).read() if st.get("model")
                   else None,
                   "model_from_stage": st.get("model_from_stage"),
                   "outputs": {}}
            for name, o in st["outputs"].items():
                if o["kind"] in ("xyz", "thermo", "restart", "text"):
                    rec["outputs"][name] = open(os.path.join(base, "goldens", case, st["name"],
                                                             name)).read()
            stages.append(rec)
        out["programs"][case] = {"potential": pot, "stages": stages}
    with open(os.path.join(HERE, "baseline_goldens.json"), "w") as f:
        json.dump(out, f, indent=1)
    os.makedirs(os.path.join(HERE, "thermostats"), exist_ok=True)
    for name in ("svr.json", "nhc.json"):
        shutil.copyfile(os.path.join(args.reference, "tests", "thermostats", "fixtures", name),
                        os.path.join(HERE, "thermostats", name))
    print("wrote", os.path.join(HERE, "baseline_goldens.json"))


if __name__ == "__main__":
    main()
