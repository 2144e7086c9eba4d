"""The nepx-md input surface (run.in, model.xyz, nep.txt header) on CPU.

`nepx-md --check` parses and validates without touching a GPU; rejected
inputs name the file and line, as the reference's parsers do
(src/run_parser.cpp, src/model_parser.cpp).
"""
import json
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

CLI = os.path.join(ROOT, "dmg-md_b200", "bin", "nepx-md")
GOLD = os.path.join(ROOT, "tests", "golden")


def _stage(tmp_path, case="single_large_nve", run_in=None, model=None):
    prog = json.load(open(os.path.join(GOLD, "baseline_goldens.json")))["programs"][case]
    st = prog["stages"][0]
    shutil.copyfile(os.path.join(GOLD, "potentials", prog["potential"]), tmp_path / "nep.txt")
    (tmp_path / "run.in").write_text(st["run_in"] if run_in is None else run_in)
    (tmp_path / "model.xyz").write_text(st["model_xyz"] if model is None else model)
    return st


def _check(tmp_path):
    if not os.path.exists(CLI):
        pytest.skip("nepx-md not built")
    return subprocess.run([CLI, "--check"], cwd=tmp_path, capture_output=True, text=True)


@pytest.mark.parametrize("case", ["single_small_static", "single_large_nve",
                                  "multi_nvt_restart", "nep_zbl_boundary"])
def test_golden_inputs_parse(tmp_path, case):
    _stage(tmp_path, case)
    r = _check(tmp_path)
    assert r.returncode == 0, r.stderr
    assert r.stdout.startswith("ok:")


@pytest.mark.parametrize("line,message", [
    ("ensemble nvt_foo 1 2 3", "unsupported command 'ensemble nvt_foo'"),
    ("ensemble nvt_ber 300 300", "ensemble nvt_ber should have 3 parameters"),
    ("ensemble nvt_ber 300 300 0.5", "temperature coupling should be >= 1"),
    ("ensemble npt_ber 300 300 100 0 100 1000 9", "isotropic 8-token syntax only"),
    ("compute_msd 10 100", "unsupported command 'compute_msd'"),
    ("frobnicate 1", "unsupported command 'frobnicate (unknown)'"),
    ("time_step abc", "time_step should be a finite real number"),
    ("dump_thermo 0", "thermo dump interval should be > 0"),
    ("dump_xyz 1 a.xyz precision triple", "invalid dump_xyz precision 'triple'"),
    ("run 1 2", "run should have 1 parameter"),
    ("velocity -3", "initial temperature should be > 0"),
])
def test_run_in_rejections(tmp_path, line, message):
    _stage(tmp_path, run_in="potential nep.txt\nensemble nve\n%s\nrun 1\n" % line)
    r = _check(tmp_path)
    assert r.returncode == 1
    assert "run.in:3" in r.stderr and message in r.stderr, r.stderr


def test_program_rules(tmp_path):
    _stage(tmp_path, run_in="potential nep.txt\ntime_step 1 0.1\nensemble nvt_bdp 300 300 100\n"
                            "run 10\n")
    r = _check(tmp_path)
    assert r.returncode == 1 and "does not support adaptive time_step" in r.stderr
    _stage(tmp_path, run_in="ensemble nve\nrun 1\n")
    r = _check(tmp_path)
    assert r.returncode == 1 and "does not contain a potential command" in r.stderr


@pytest.mark.parametrize("body", [
    "time_step 1 0.05\nensemble nve\nrun 10\n",
    "time_step 1 0.05\nensemble nvt_ber 300 300 100\nrun 10\n",
    "ensemble nve\ncorrect_velocity 10\nrun 20\n",
    "ensemble nvt_ber 300 300 100\ncorrect_velocity 10 0\nrun 20\n",
    "ensemble nve\ndump_xyz 5 a.xyz unwrapped_position velocity\nrun 10\n",
])
def test_run_in_md_controls_accepted(tmp_path, body):
    """correct_velocity, the adaptive time step and unwrapped positions run
    with the ensembles the reference allows them with."""
    _stage(tmp_path, run_in="potential nep.txt\n" + body)
    r = _check(tmp_path)
    assert r.returncode == 0, r.stderr


@pytest.mark.parametrize("body,message", [
    ("ensemble npt_ber 300 300 100 0 100 1000\ncorrect_velocity 10\nrun 10\n",
     "ensemble npt_ber does not support correct_velocity"),
    ("time_step 1 0.05\nensemble nvt_nhc 300 300 100\nrun 10\n",
     "ensemble nvt_nhc does not support adaptive time_step"),
    ("ensemble nve\ncorrect_velocity 5\nrun 10\n",
     "velocity correction interval should be >= 10"),
])
def test_run_in_md_controls_rules(tmp_path, body, message):
    _stage(tmp_path, run_in="potential nep.txt\n" + body)
    r = _check(tmp_path)
    assert r.returncode == 1 and message in r.stderr, r.stderr


@pytest.mark.parametrize("edit,message", [
    (lambda m: m.replace("Lattice=\"24 0 0 0 24 0 0 0 24\"", "Lattice=\"24 0 0 0 24 0\""),
     "Lattice should contain nine values"),
    (lambda m: m.replace("C 8.0", "Si 8.0", 1), "species 'Si' is not allowed by the potential"),
    (lambda m: "1\n" + m.split("\n", 1)[1], "number of atoms should be >= 2"),
    (lambda m: m.replace("pbc=\"T T T\"", "pbc=\"T T X\""), "pbc should contain only T or F"),
])
def test_model_rejections(tmp_path, edit, message):
    st = _stage(tmp_path)
    (tmp_path / "model.xyz").write_text(edit(st["model_xyz"]))
    r = _check(tmp_path)
    assert r.returncode == 1 and message in r.stderr, r.stderr


@pytest.mark.parametrize("line,ok", [
    ("ensemble npt_ber 300 300 100 0 0 0 100 120 140 1000", True),
    ("ensemble npt_scr 300 300 100 0 0 0 0 0 0 100 100 100 50 50 50 1000", True),
    ("ensemble npt_ber 300 300 100 0 0 0 100 120 -140 1000", False),
    ("ensemble npt_ber 300 300 100 0 0 0 100 120 140 1000 7", False),
    ("ensemble npt_ber 300 300 100 0 0 0 0 100 120 140 1000", False),
])
def test_component_barostat_syntax(tmp_path, line, ok):
    """The anisotropic (12-token) and triclinic (18-token) npt forms."""
    _stage(tmp_path, run_in="potential nep.txt\nvelocity 300\ntime_step 1\n%s\nrun 10\n" % line)
    r = _check(tmp_path)
    assert (r.returncode == 0) == ok, r.stderr
