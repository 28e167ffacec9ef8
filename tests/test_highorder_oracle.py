"""The oracle's restatement of the high-order path (tioga.C:162-178,
highOrder.C) against the compiled reference, both driven by the same
Lagrange-hex callbacks (oracle/ho_callbacks.c).  CPU only.

The reference's callbacks carry no block id, so this pins the oracle on a
configuration where only one block ever plays each role: the shell has no
wall (no holes) and the background's user resolution is so fine that none of
its nodes becomes a receptor.  The shell's points are then searched in the
background only."""
import os

import numpy as np
import pytest

from tioga_b200 import cases
from tests.ho_harness import run_highorder, diff_highorder

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE = os.path.join(ROOT, "oracle", "_ref", "liboracle.so")
REF = os.path.join(ROOT, "oracle", "_ref", "libtioga_ref.so")


@pytest.mark.skipif(not (os.path.exists(ORACLE) and os.path.exists(REF)),
                    reason="needs the oracle and the compiled reference (make -C oracle)")
@pytest.mark.parametrize("seed", [4, 9])
def test_highorder_oracle_matches_reference(seed):
    system, ho = cases.small_config4(seed, wall=False)
    nvar = 3
    q = cases.dof_fields(ho, nvar, seed=seed)
    bg = system.blocks[0]
    res = {bg.tag: (np.full(bg.nnodes, 1e-6), np.full(bg.ncells, 1e-6))}
    a = run_highorder(ORACLE, system, ho, nvar, q, "hook", resolutions=res)
    b = run_highorder(REF, system, ho, nvar, q, "roles", resolutions=res)
    assert not diff_highorder(system, a, b, points=False)
    shell = system.blocks[1]
    changed = int((a["q"][shell.tag] != q[1]).sum())
    assert changed > 0  # the receptor cells' DOFs were interpolated
    assert (a["cells"][shell.tag] == -1).sum() > 0
