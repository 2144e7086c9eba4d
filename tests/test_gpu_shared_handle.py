"""One handle, two users: an MD that shares its potential handle with direct
force calls on another system between its runs continues as an MD that had
the handle to itself: its Verlet rows and box are rebuilt for it when it
takes the handle back.  The agreement is to FP32 rounding, not bitwise: the
typewise filter sums the radial descriptors over the Verlet candidates in
lane order, and the candidate set depends on when the list was last built.
A stale list or box would give errors of order one."""
import numpy as np
import pytest

import workloads
from conftest import potential

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp32", "mixed"])
def test_md_continues_after_another_caller(precision):
    import nepx
    path = potential("nep_water.txt")
    t, h, p = workloads.water(n_mol=200, seed=51)
    masses = np.where(np.asarray(t) == 0, 15.999, 1.008)
    v = workloads.maxwell_boltzmann(masses, 300.0, seed=52)
    to, ho, po = workloads.water(n_mol=500, seed=53)   # the other caller's system
    rows = []
    # one handle for both runs: its autotuned lane grouping (which sets the
    # FP32 summation order) is then the same
    pot = nepx.Potential(path, max_atoms=2000)
    pot.set_precision(precision)
    for interleave in (False, True):
        md = nepx.MD(pot, t, masses, p, v, h)
        md.set_ensemble("nvt_ber", T0=300.0, Tdamp=100.0)
        r1 = md.run(30, 0.5, thermo_every=10)
        if interleave:
            tt = torch.as_tensor(np.asarray(to, dtype=np.int32), device="cuda")
            pp = torch.as_tensor(np.ascontiguousarray(po), device="cuda")
            pot.compute(tt, ho, pp, sync_check=True)
        r2 = md.run(30, 0.5, thermo_every=10)
        rows.append(np.concatenate([r1, r2]))
        md.close()
    pot.close()
    a, b = rows
    # per column, against the column's scale (temperature, energies, stresses, box).
    # The rebuilt Verlet rows hand the radial edges to other lanes, which moves
    # FP32 sums by an ulp; on the mixed path such an ulp can move a 16-bit ANN
    # operand by one unit (2^-11 relative), hence the looser bound there
    scale = np.abs(a).max(axis=0) + 1e-12
    rel = (np.abs(a - b) / scale).max()
    assert rel <= (1e-5 if precision == "fp32" else 3e-4), rel
