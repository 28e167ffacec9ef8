"""Batched form on the GPU: many independent overset systems registered in one
instance (tioga_b200_registergrid_sys_) and connected by one preprocess, one
connectivity and one data update.  Every system's iblanks, donor lists,
weights and updated fields must equal, bit for bit, what the oracle gives for
that system alone (the reference runs systems one after another,
driver/poisson_mms.f90:111-253)."""
import copy

import numpy as np
import pytest

import tioga_b200 as tb
from tioga_b200 import cases
from tioga_b200.capi import TiogaLibrary, run_batch, run_system
from tests.compare import diff_runs

pytestmark = pytest.mark.gpu


def _systems():
    out = cases.small_config2(2, nsys=6)
    out.insert(2, cases.small_config0_seam(4))  # coincident query points in the middle of the batch
    return out


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "split"])
def test_batch_equals_each_system_alone(precision, oracle_lib):
    systems = _systems()
    qs = [cases.fields(s, nvar=5, seed=20 + k) for k, s in enumerate(systems)]

    def setup(t):
        tb.set_int(t.lib, "tioga_b200_set_precision_", precision)
        assert t.lib.tioga_b200_nsystems_() == len(systems)

    outs = run_batch(tb.library_path(), systems, q_sets=qs, setup=setup)
    for k, system in enumerate(systems):
        ref = run_system(oracle_lib, system, q_blocks=qs[k])
        problems = diff_runs(system, ref, outs[k])
        assert not problems, f"system {k} ({system.name}):\n" + "\n".join(problems)


def _rigid(system, seed):
    """The shells of a system rotated by up to 2 degrees about a random axis
    and moved by a small translation (a moving-body time step)."""
    rng = np.random.default_rng(seed)
    out = copy.deepcopy(system)
    for b in out.blocks[1:]:
        ax = rng.normal(size=3)
        ax /= np.linalg.norm(ax)
        th = np.deg2rad(rng.uniform(0.0, 2.0))
        K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
        R = np.eye(3) + np.sin(th) * K + (1 - np.cos(th)) * (K @ K)
        c = b.x.mean(axis=0)
        b.x[:] = (b.x - c) @ R.T + c + rng.uniform(-0.02, 0.02, 3)
    return out


def test_batch_second_call_after_motion(oracle_lib):
    """Two connectivity calls of one batch instance, the shells of every
    system moved in between: the second call's results equal fresh runs of
    the moved systems alone (every system's donor state is undone)."""
    systems = _systems()
    moved = [_rigid(s, 50 + k) for k, s in enumerate(systems)]
    t = TiogaLibrary(tb.library_path())
    t.init()
    t.register_batch(systems)
    t.preprocess_grids()
    t.performconnectivity()
    for k, s in enumerate(moved):  # the registered coordinate arrays are the library's view
        for b in s.blocks:
            t.blocks[(k, b.tag)]["x"][:] = b.x.reshape(-1)
    t.preprocess_grids()
    t.performconnectivity()
    assert t.lib.tioga_b200_last_error() == 0
    for k, s in enumerate(moved):
        t.select_system(k)
        got = {"iblank": {}, "donors": {}, "q": {}}
        for b in s.blocks:
            got["iblank"][b.tag] = t.blocks[(k, b.tag)]["iblank"].copy()
            got["donors"][b.tag] = t.getdonorinfo(b.tag)
        ref = run_system(oracle_lib, s)
        problems = diff_runs(s, ref, got)
        assert not problems, f"system {k} ({s.name}):\n" + "\n".join(problems)
    t.delete()
