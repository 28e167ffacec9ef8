"""Edge cases of the connectivity call: blocks that do not overlap at all (no
block pairs, no queries), a single block, a shell without wall nodes (no hole
map), and a shell whose wall is its only boundary.  On the CPU the oracle is
checked against the compiled reference on each; on the GPU the library is
checked against the oracle.  Bar: identical iblanks, donor lists, weights
and updated fields."""
import copy
import os

import numpy as np
import pytest

from tests.compare import diff_runs
from tests.conftest import REF_LIB
from tioga_b200 import cases
from tioga_b200.capi import run_system


def _far_apart():
    s = cases.small_config0(0)
    s = copy.deepcopy(s)
    s.blocks[1].x[:, 0] += 100.0  # the shell far outside the background
    return s


def _single_block():
    s = cases.small_config1(1)
    return cases.System([copy.deepcopy(s.blocks[0])], "single block")


def _no_wall():
    s = copy.deepcopy(cases.small_config0(0))
    b = s.blocks[1]
    s.blocks[1] = cases.Block(b.tag, b.x, b.cells, np.zeros(0, np.int32), b.obc, b.name)
    return s


def _no_obc():
    s = copy.deepcopy(cases.small_config1(2))
    b = s.blocks[2]
    s.blocks[2] = cases.Block(b.tag, b.x, b.cells, b.wbc, np.zeros(0, np.int32), b.name)
    return s


EDGE = {"far-apart": _far_apart, "single-block": _single_block, "no-wall": _no_wall, "no-obc": _no_obc}


def _run(lib, system):
    q = cases.fields(system, nvar=2, seed=5)
    return run_system(lib, system, q_blocks=q, nvar=2)


@pytest.mark.parametrize("name", list(EDGE))
def test_oracle_matches_compiled_reference(name, oracle_lib):
    if not os.path.exists(REF_LIB):
        pytest.skip("the compiled reference needs the reference sources (make -C oracle ref)")
    system = EDGE[name]()
    ref, got = _run(REF_LIB, system), _run(oracle_lib, system)
    problems = diff_runs(system, ref, got)
    assert not problems, "\n".join(problems)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(EDGE))
def test_gpu_matches_oracle(name, oracle_lib):
    from tioga_b200 import extras, library_path, stats

    def after(t):
        extras(t.lib)
        assert t.lib.tioga_b200_last_error() == 0
        return stats(t.lib)

    system = EDGE[name]()
    q = cases.fields(system, nvar=2, seed=5)
    ref = run_system(oracle_lib, system, q_blocks=q, nvar=2)
    got = run_system(library_path(), system, q_blocks=q, nvar=2, after=after)
    problems = diff_runs(system, ref, got)
    assert not problems, "\n".join(problems)
    if name in ("far-apart", "single-block"):
        assert got["after"]["nquery"] == 0
