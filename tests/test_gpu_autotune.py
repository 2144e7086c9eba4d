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
    assert len(fields) == 19
    import numpy as np
    assert np.array_equal(np.load(forces[0]), np.load(forces[1]))
