"""The autotuner's picks are kept per (device, model shape, precision, row
path, size class): a second handle of the same process, and with
NEPX_TUNE_FILE a later process, reuse them without timing the variants again,
and the results are the same bit for bit (the picks set the lane grouping,
hence the FP32 summation order)."""
import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

SCRIPT = r"""
import sys
sys.path.insert(0, %r); sys.path.insert(0, %r)
import numpy as np, torch, workloads, nepx
from conftest import potential
t, h, p = workloads.water(n_mol=700, seed=4)
tt = torch.as_tensor(t, device="cuda"); pp = torch.as_tensor(p, device="cuda")
out = []
for k in range(2):
    pot = nepx.Potential(potential("nep_water.txt"), max_atoms=len(t))
    pe, f, w = pot.compute(tt, h, pp, sync_check=True)
    out.append(f.cpu().numpy())
    pot.close()
assert np.array_equal(out[0], out[1])
np.save(sys.argv[1], out[0])
"""


def test_tune_file_reused_across_processes(tmp_path):
    tune = tmp_path / "tune.txt"
    env = dict(os.environ, NEPX_TUNE_FILE=str(tune))
    code = SCRIPT % (os.path.join(ROOT, "dmg-md_b200"), os.path.join(ROOT, "tests"))
    forces = []
    lines = []
    for k in range(2):
        target = tmp_path / ("f%d.npy" % k)
        r = subprocess.run([sys.executable, "-c", code, str(target)], env=env, cwd=ROOT,
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        lines.append(tune.read_text().splitlines())
        forces.append(target)
    # the first process tuned once (its second handle reused the pick), the
    # second process found it in the file
    assert len(lines[0]) == 1 and lines[1] == lines[0]
    fields = lines[0][0].split()
    assert len(fields) == 21   # 14 key fields, 7 launch choices
    import numpy as np
    assert np.array_equal(np.load(forces[0]), np.load(forces[1]))


# ---- pinned launch choices ------------------------------------------------

def _systems(tmp_path):
    """Models of the shape the fused angular force serves (n_max <= 4, basis
    <= 8, l_max <= 4): the water potential and the benchmark's synthetic
    carbon NEP4, on large boxes."""
    import workloads
    from conftest import potential
    t, h, p = workloads.water(n_mol=700, seed=5)
    yield "water", potential("nep_water.txt"), t, h, p
    path = workloads.write_nep(str(tmp_path / "c.txt"), version=4, symbols=("C",),
                               rc=(4.2, 3.7), mn=(100, 60), n_max=(4, 4), basis=(8, 8),
                               l_max=(4, 2, 1), H=30, seed=2025, q_scaler=0.02)
    t, h, p = workloads.diamond(ncell=5, jitter=0.08, seed=6)
    yield "carbon", path, t, h, p


def test_every_launch_choice_matches_oracle(tmp_path):
    """Each lane grouping, occupancy build (descriptor kernel and gather) and
    both forms of the angular force (own kernel, or inside the descriptor
    kernel), pinned with
    nepx_set_tuning, against the FP64 oracle at the FP32 tolerances; the
    mixed-precision build with the fused angular force at its own."""
    import numpy as np
    import torch
    import nepx
    import oracle
    from test_gpu_force import assert_close
    from test_gpu_mixed import assert_mixed_close
    for name, path, t, h, p in _systems(tmp_path):
        ref = oracle.OracleModel(path).compute(t, h, p)
        tt = torch.as_tensor(np.asarray(t, dtype=np.int32), device="cuda")
        pp = torch.as_tensor(np.ascontiguousarray(p), device="cuda")
        pot = nepx.Potential(path, max_atoms=len(t))
        for ff in (0, 1):
            for g in (4, 8):
                for ctas in (3, 4):
                    pot.set_tuning(filter_group=g, fused_group=g, fused_ctas_per_sm=ctas,
                                   f12_group=12 - g, gather_group=g, fused_f12=ff,
                                   gather_ctas_per_sm=7 - ctas)
                    got = [x.cpu().numpy() for x in pot.compute(tt, h, pp, sync_check=True)]
                    assert pot.tuning() == ({"filter_group": g, "fused_group": g,
                                             "fused_ctas_per_sm": ctas, "f12_group": 12 - g,
                                             "gather_group": g, "fused_f12": ff,
                                             "gather_ctas_per_sm": 7 - ctas}, True)
                    assert_close(ref, got, "%s ff=%d G=%d ctas=%d" % (name, ff, g, ctas))
        pot.set_precision("mixed")
        pot.set_tuning(fused_f12=1, fused_group=4)
        got = [x.cpu().numpy() for x in pot.compute(tt, h, pp, sync_check=True)]
        assert_mixed_close(ref, got, name + " fused f12", "mixed")
        with pytest.raises(nepx.NepxError):
            pot.set_tuning(fused_group=5)
        pot.close()


def test_autotuner_times_the_fused_angular_force(tmp_path):
    """With nothing pinned the first compute fixes every choice, and the
    chosen form gives the oracle's forces."""
    import numpy as np
    import torch
    import nepx
    import oracle
    from test_gpu_force import assert_close
    name, path, t, h, p = next(_systems(tmp_path))
    pot = nepx.Potential(path, max_atoms=len(t))
    assert pot.tuning()[1] is False
    tt = torch.as_tensor(np.asarray(t, dtype=np.int32), device="cuda")
    pp = torch.as_tensor(np.ascontiguousarray(p), device="cuda")
    got = [x.cpu().numpy() for x in pot.compute(tt, h, pp, sync_check=True)]
    choice, tuned = pot.tuning()
    assert tuned and choice["fused_f12"] in (0, 1)
    assert_close(oracle.OracleModel(path).compute(t, h, p), got, name)
    pot.close()
