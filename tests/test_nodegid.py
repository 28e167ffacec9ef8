"""The node-global-id variant (TIOGA_HAS_NODEGID): blocks carry node global
ids, and coincident query points of a donor are merged by id
(uniquenode_map, src/search.C:48-74, selected at :242-246) instead of by the
octree over their coordinates.  The reference switches it at compile time;
oracle/Makefile builds the reference that way too (_ref/libtioga_ref_nodegid.so,
registration through the test shim's refshim_registergrid_gids_).

The seam meshes duplicate their phi seams: every seam node has a twin at the
same place, and the twins share a global id, as copies of one node on two
partitions do.  CPU: the oracle's restatement against the compiled reference.
GPU: the library (tioga_b200_registernodegid_, tioga_b200_set_nodegid_merge_)
against the compiled reference, in both precision forms."""
import ctypes as C
import os

import numpy as np
import pytest

from tioga_b200 import cases
from tioga_b200.capi import run_system
from tests.compare import diff_runs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_NG = os.path.join(ROOT, "oracle", "_ref", "libtioga_ref_nodegid.so")

SYSTEMS = {
    "cfg1_seam_s1": lambda: cases.small_config1_seam(1),
    "cfg0_seam_s2": lambda: cases.small_config0_seam(2),
    "cfg1_s1": lambda: cases.small_config1(1),
    # twins with ids of their own: the id merge keeps them apart, where the
    # octree would merge them; the shells' resolutions make that visible
    "cfg0_seam_s2_own_ids": lambda: cases.small_config0_seam(2),
}


def node_gids(system, share=True):
    """Per block: tag << 40 plus the node's index, coincident nodes (the seam
    twins) sharing the id of the first of them when `share`."""
    out = []
    for b in system.blocks:
        if share:
            _, first, inv = np.unique(np.round(b.x, 10), axis=0, return_index=True, return_inverse=True)
            ids = first[inv.reshape(-1)]
        else:
            ids = np.arange(b.nnodes)
        out.append((np.uint64(b.tag) << np.uint64(40)) + ids.astype(np.uint64))
    return out


def _inputs(name):
    system = SYSTEMS[name]()
    gids = node_gids(system, share=not name.endswith("own_ids"))
    res = None
    if name.endswith("own_ids"):
        rng = np.random.default_rng(98)
        res = {b.tag: (rng.uniform(0.02, 0.6, b.nnodes), rng.uniform(0.02, 0.6, b.ncells)) for b in system.blocks[1:]}
    return system, gids, res


def _merge_on(kind):
    def setup(t):
        if kind == "oracle":
            t.lib.tioga_oracle_set_nodegid_merge(C.c_int(1))
        elif kind == "gpu":
            t.lib.tioga_b200_set_nodegid_merge_(C.byref(C.c_int(1)))
    return setup


def test_seam_twins_share_ids():
    s = cases.small_config1_seam(1)
    g = node_gids(s)
    assert sum(int(b.nnodes - np.unique(x).size) for b, x in zip(s.blocks, g)) > 0


@pytest.mark.skipif(not os.path.exists(REF_NG), reason="needs the node-GID reference (make -C oracle ref_nodegid)")
@pytest.mark.parametrize("name", list(SYSTEMS))
def test_oracle_nodegid_matches_reference(oracle_lib, name):
    system, gids, res = _inputs(name)
    q = cases.fields(system, nvar=4, seed=61)
    ref = run_system(REF_NG, system, q_blocks=q, nvar=4, node_gids=gids, resolutions=res)
    orc = run_system(oracle_lib, system, q_blocks=q, nvar=4, node_gids=gids, resolutions=res,
                     setup=_merge_on("oracle"))
    assert not diff_runs(system, ref, orc)
    if name.endswith("own_ids"):  # the case is live: the octree merge gives another result
        octree = run_system(oracle_lib, system, q_blocks=q, nvar=4, resolutions=res)
        assert diff_runs(system, octree, ref)


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF_NG), reason="needs the node-GID reference (make -C oracle ref_nodegid)")
@pytest.mark.parametrize("name", list(SYSTEMS))
@pytest.mark.parametrize("precision", [1, 0])
def test_gpu_nodegid_matches_reference(name, precision):
    import tioga_b200 as tb
    system, gids, res = _inputs(name)
    q = cases.fields(system, nvar=4, seed=61)
    ref = run_system(REF_NG, system, q_blocks=q, nvar=4, node_gids=gids, resolutions=res)

    def setup(t):
        _merge_on("gpu")(t)
        tb.set_int(t.lib, "tioga_b200_set_precision_", precision)

    gpu = run_system(tb.library_path(), system, q_blocks=q, nvar=4, node_gids=gids, resolutions=res, setup=setup,
                     after=lambda t: (tb.extras(t.lib).tioga_b200_last_error(), tb.stats(t.lib)["nmerged"]))
    assert gpu["after"][0] == 0
    if "seam" in name and not name.endswith("own_ids"):
        assert gpu["after"][1] > 0  # twins were merged
    assert not diff_runs(system, ref, gpu)
