"""A run that writes a restart and goes on equals, bit for bit, a run
restarted from those files (state, time, step, DtMax_B), in the 'one' and
'block' layouts, on a uniform and on a block-adaptive grid."""
import numpy as np
import pytest

from batsrus_b200 import configs, initial, restart
from batsrus_b200.explicit import ExplicitSolver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,grid", [("one", "ot"), ("block", "blast")])
def test_restart_continues_bit_exactly(tmp_path, kind, grid):
    if grid == "ot":
        g, s, st, _ = configs.uniform_3d_case(2, "Linde", "mc3", 1.2, state="blast")
    else:
        g, s, st, _ = configs.amr_blast(nRoot=2, maxLevel=2, precision="fp64")
    x = ExplicitSolver(g, s)
    x.set_state(st)
    x.advance(3)
    restart.write_restart(str(tmp_path), x, kind)
    x.advance(3)
    ref, tref = x.get_state(), x.time()
    x.close()
    y = restart.restart_solver(str(tmp_path), s)
    assert y.time()[2] == 3
    y.advance(3)
    isl = y.grid.interior_slices()
    assert np.array_equal(y.get_state()[isl], ref[isl])
    assert y.time() == tref
    y.close()
