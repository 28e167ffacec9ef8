"""GPU parity: the B200 library against the oracle (the C restatement of the
reference, itself pinned bit for bit to the compiled reference), through the
same TIOGA C ABI on the same seeded inputs.

Bar: iblank, receptor lists and donor cell/node indices identical; weights
and the updated fields identical bit for bit (the FP64 arithmetic follows the
reference's operation order, compiled without FMA contraction).  The only
allowed difference is a donor that depends on the reference's tree visiting
order (several cells accept the point, or a point on the face of a no-donor
cell); the library counts those, and these inputs have none."""
import ctypes as C

import numpy as np
import pytest

import tioga_b200 as tb
from tioga_b200 import cases
from tioga_b200.capi import run_system
from tests.compare import diff_runs

pytestmark = pytest.mark.gpu

CASES = {
    "cfg0-small": lambda: cases.small_config0(0),
    "cfg0-small-seed5": lambda: cases.small_config0(5),
    "cfg1-small": lambda: cases.small_config1(1),
    "cfg1-small-seed3": lambda: cases.small_config1(3),
    "cfg0": lambda: cases.config0(0),
    "cfg0-small-seam": lambda: cases.small_config0_seam(0),
    "cfg1-small-seam": lambda: cases.small_config1_seam(1),
}


def _gpu_setup(precision):
    def setup(t):
        tb.set_int(t.lib, "tioga_b200_set_precision_", precision)
    return setup


def _gpu_after(t):
    tb.extras(t.lib)
    assert t.lib.tioga_b200_last_error() == 0
    return tb.stats(t.lib)


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "split"])
@pytest.mark.parametrize("name", list(CASES))
def test_parity_with_oracle(name, precision, oracle_lib):
    system = CASES[name]()
    q = cases.fields(system, nvar=5, seed=11)
    ref = run_system(oracle_lib, system, q_blocks=q)
    gpu = run_system(tb.library_path(), system, q_blocks=q, setup=_gpu_setup(precision), after=_gpu_after)
    st = gpu["after"]
    assert st["error"] == 0, st
    assert st["nties"] == 0, st
    problems = diff_runs(system, ref, gpu)
    assert not problems, "\n".join(problems)
    # the duplicated seams give coincident query points, which must be merged
    assert (st["nmerged"] > 0) == name.endswith("seam"), st


@pytest.mark.parametrize("itype", ["row", "column"])
def test_dataupdate_layouts(itype, oracle_lib):
    system = cases.small_config1(2)
    nvar = 3
    q = cases.fields(system, nvar=nvar, seed=4)
    ref = run_system(oracle_lib, system, q_blocks=q, nvar=nvar, itype=itype)
    gpu = run_system(tb.library_path(), system, q_blocks=q, nvar=nvar, itype=itype)
    assert not diff_runs(system, ref, gpu)


@pytest.mark.parametrize("opts", [dict(isym=0), dict(isym=1), dict(isym=2), dict(nfringe=2),
                                  dict(nfringe=0), dict(mexclude=0), dict(mexclude=1)],
                         ids=lambda d: ",".join(f"{k}={v}" for k, v in d.items()))
def test_settings(opts, oracle_lib):
    system = cases.small_config0(1)
    q = cases.fields(system, nvar=2, seed=3)
    ref = run_system(oracle_lib, system, q_blocks=q, nvar=2, **opts)
    gpu = run_system(tb.library_path(), system, q_blocks=q, nvar=2, **opts)
    assert not diff_runs(system, ref, gpu)


def test_linear_field_exact():
    """The reference driver's known answer (driver/testTioga.f90:145-166):
    q = x+y+z is reproduced at every receptor to round-off."""
    system = cases.config0(0)
    q = cases.linear_fields(system, nvar=5)
    gpu = run_system(tb.library_path(), system, q_blocks=q)
    for b in system.blocks:
        exact = b.x.sum(axis=1)
        err = np.abs(gpu["q"][b.tag].reshape(-1, 5) - exact[:, None]).max()
        assert err < 1e-12
        assert (gpu["iblank"][b.tag] == -1).sum() > 0


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "split"])
@pytest.mark.parametrize("name", ["cfg0_small_s0", "cfg1_small_s1", "cfg0_small_s1_opts",
                                  "cfg1_small_s2_userres", "cfg0_small_s0_reduce", "cfg1_small_s1_reduce_nf2",
                                  "cfg1_small_s1_seam_reduce"])
def test_gpu_matches_reference_fixtures(name, precision):
    """The GPU library against the compiled reference's own outputs."""
    from tests.golden import make_golden as mg
    from tests.test_oracle_golden import load
    g = load(name)
    fac, _, nvar, itype, fseed = mg.CASES[name]
    system = fac()
    assert str(g["digest"]) == mg.digest(system)
    q = cases.fields(system, nvar=nvar, seed=fseed)
    out = run_system(tb.library_path(), system, q_blocks=q, nvar=nvar, itype=itype,
                     setup=_gpu_setup(precision), **mg.settings_for(name, system))
    for b, q0 in zip(system.blocks, q):
        t = b.tag
        np.testing.assert_array_equal(out["iblank"][t], g[f"iblank_{t}"].astype(np.int32))
        rec, ind, frac = out["donors"][t]
        np.testing.assert_array_equal(rec, g[f"receptors_{t}"])
        np.testing.assert_array_equal(ind, g[f"indices_{t}"])
        assert np.array_equal(frac.view(np.int64), g[f"frac_{t}"].view(np.int64))
        changed = np.nonzero(out["q"][t] != q0)[0]
        np.testing.assert_array_equal(changed, g[f"qidx_{t}"])
        assert np.array_equal(out["q"][t][changed].view(np.int64), g[f"qval_{t}"].view(np.int64))


@pytest.mark.parametrize("name", ["cfg0-small", "cfg1-small", "cfg0"])
def test_query_count_matches_oracle(name, oracle_lib):
    """Q, the metric's unit (query points handed to donor searches), against
    the reference's nsearch totals, and every block's cell iblank.

    Q depends on the blocks' oriented boxes, which only cull.  Their axes are
    covariance eigenvectors; the reference sums sequentially and the GPU in a
    reduction tree, so the last bits differ.  On the jittered cfg0 meshes that
    changes nothing and Q must be equal.  The unjittered cfg1 lattice has an
    exactly isotropic covariance and each shell a degenerate eigenvalue pair,
    so there the axes within the degenerate subspace are set by rounding noise
    and Q may differ by a few per cent; the connectivity results are the same
    either way (every other test here)."""
    import ctypes as C
    from tioga_b200.capi import TiogaLibrary
    system = CASES[name]()
    counts = {}
    cells = {}
    for path in (oracle_lib, tb.library_path()):
        t = TiogaLibrary(path)
        t.init()
        t.register_system(system)
        t.preprocess_grids()
        t.performconnectivity()
        if path == oracle_lib:
            ns, nd, tot = C.c_int(), C.c_int(), 0
            for b in system.blocks:
                t.lib.tioga_oracle_searchstats(C.c_int(b.tag), C.byref(ns), C.byref(nd))
                tot += ns.value
            counts["oracle"] = tot
            for b in system.blocks:
                out = np.zeros(b.ncells, np.int32)
                t.lib.tioga_oracle_getcelliblank(C.c_int(b.tag), out.ctypes.data_as(C.c_void_p))
                cells[("oracle", b.tag)] = out
        else:
            tb.extras(t.lib)
            counts["gpu"] = tb.stats(t.lib)["nquery"]
            for b in system.blocks:
                out = np.zeros(b.ncells, np.int32)
                t.lib.tioga_b200_getcelliblank_(C.byref(C.c_int(b.tag)), out.ctypes.data_as(C.c_void_p))
                cells[("gpu", b.tag)] = out
        t.delete()
    for b in system.blocks:
        g, o = cells[("gpu", b.tag)], cells[("oracle", b.tag)]
        bad = np.flatnonzero(g != o)
        assert bad.size == 0, (b.tag, bad.size, bad[:8], g[bad[:8]], o[bad[:8]])
    if name.startswith("cfg0"):
        assert counts["gpu"] == counts["oracle"], counts
    else:
        assert abs(counts["gpu"] - counts["oracle"]) <= 0.02 * counts["oracle"], counts


def _two_calls(lib_path, system, shift, extras_fn, setup=None):
    """preprocess, connectivity, move the last block by `shift` in the
    caller's own coordinate array (the library reads it again), connectivity
    again; returns iblanks, donor info and cell iblanks after each call."""
    import copy
    from tioga_b200.capi import TiogaLibrary
    system = copy.deepcopy(system)  # the library keeps (and this moves) the caller's arrays
    t = TiogaLibrary(lib_path)
    t.init()
    t.register_system(system)
    if setup is not None:
        setup(t)
    t.preprocess_grids()
    outs = []
    for call in range(2):
        if call == 1:
            x = t.blocks[system.blocks[-1].tag]["x"].reshape(-1, 3)
            x += np.asarray(shift)
        t.performconnectivity()
        out = {"iblank": {}, "donors": {}, "q": {}, "cells": {}}
        for b in system.blocks:
            out["iblank"][b.tag] = t.iblank(b.tag).copy()
            out["donors"][b.tag] = t.getdonorinfo(b.tag)
            cell = np.zeros(b.ncells, np.int32)
            extras_fn(t.lib, b.tag, cell)
            out["cells"][b.tag] = cell
        outs.append(out)
    t.delete()
    return outs


@pytest.mark.parametrize("name", ["cfg0-small", "cfg1-small"])
@pytest.mark.parametrize("precision", [0, 1])
def test_second_call_after_motion(name, precision, oracle_lib):
    """A second connectivity call after the shell moved (no new preprocess,
    as a solver between time steps) gives the reference's answer: the holes,
    receptors and cell iblanks of the first call are undone and rebuilt."""
    import ctypes as C
    system = CASES[name]()
    h = (system.blocks[0].x.max() - system.blocks[0].x.min()) / round(system.blocks[0].nnodes ** (1 / 3))
    shift = (0.31 * h, -0.17 * h, 0.23 * h)  # a fraction of a background cell

    def oracle_cells(lib, tag, out):
        lib.tioga_oracle_getcelliblank(C.c_int(tag), out.ctypes.data_as(C.c_void_p))

    def gpu_cells(lib, tag, out):
        lib.tioga_b200_getcelliblank_(C.byref(C.c_int(tag)), out.ctypes.data_as(C.c_void_p))

    ref = _two_calls(oracle_lib, system, shift, oracle_cells)
    gpu = _two_calls(tb.library_path(), system, shift, gpu_cells, _gpu_setup(precision))
    for call in range(2):
        bad = diff_runs(system, ref[call], gpu[call])
        assert not bad, (call, bad)
        for b in system.blocks:
            np.testing.assert_array_equal(gpu[call]["cells"][b.tag], ref[call]["cells"][b.tag])
    moved = sum(int((ref[0]["iblank"][b.tag] != ref[1]["iblank"][b.tag]).sum()) for b in system.blocks)
    assert moved > 0  # the motion changed the answer, so the second call is a real test


def test_autotune_keeps_results():
    """The autotuner only changes launch shapes: after it the connectivity
    results are the same bits, and the chosen shapes are among its choices."""
    import ctypes as C
    from tioga_b200.capi import TiogaLibrary
    system = cases.small_config1(3)
    t = TiogaLibrary(tb.library_path())
    tb.extras(t.lib)
    t.init()
    t.register_system(system)
    t.preprocess_grids()
    t.performconnectivity()
    before = {b.tag: (t.iblank(b.tag).copy(), t.getdonorinfo(b.tag)) for b in system.blocks}
    tb.set_int(t.lib, "tioga_b200_autotune_", 1)
    assert t.lib.tioga_b200_last_error() == 0
    out = (C.c_int * 8)()
    t.lib.tioga_b200_tuning_(out)
    assert out[0] in (2, 3, 4) and out[1] in (32, 64, 128) and out[2] in (4, 8, 16, 32, 64)
    assert out[3] in (16, 32, 64, 128) and out[4] in (8, 16, 32, 64)
    assert out[5] in (4, 6, 8) and out[6] in (0, 1)
    for b in system.blocks:
        ib, (r, i, f) = before[b.tag]
        r2, i2, f2 = t.getdonorinfo(b.tag)
        assert np.array_equal(ib, t.iblank(b.tag))
        assert np.array_equal(r, r2) and np.array_equal(i, i2)
        assert np.array_equal(f.view(np.int64), f2.view(np.int64))
    t.delete()


@pytest.mark.parametrize("name", ["cfg0", "cfg1-small-seed3"])
@pytest.mark.parametrize("variant", [1, 2])
def test_traversal_variants_match_oracle(name, variant, oracle_lib):
    """Both traversals of the split form (leaves tested as met, and leaves
    postponed until every lane of a warp holds one) give the oracle's results."""
    import ctypes as C
    system = CASES[name]()
    q = cases.fields(system, nvar=3, seed=17)

    def setup(t):
        _gpu_setup(1)(t)
        t.lib.tioga_b200_set_tuning_((C.c_int * 7)(0, 0, 0, 0, 0, 0, variant))

    def variant_in_use(t):
        out = (C.c_int * 8)()
        tb.extras(t.lib).tioga_b200_tuning_(out)
        return out[6]

    ref = run_system(oracle_lib, system, q_blocks=q, nvar=3)
    gpu = run_system(tb.library_path(), system, q_blocks=q, nvar=3, setup=setup, after=variant_in_use)
    assert gpu["after"] == variant - 1
    problems = diff_runs(system, ref, gpu)
    assert not problems, "\n".join(problems)


@pytest.mark.parametrize("chunk", [4096, 65537])
def test_chunked_upload_matches_oracle(chunk, oracle_lib):
    """The split form uploads the coordinates in chunks and makes each chunk's
    cell boxes as it lands.  With chunks far smaller than the default, cfg0's
    background spans many chunks and a chunk spans the background's end and
    the shell's start; the results equal the oracle's."""
    import ctypes as C
    system = CASES["cfg0"]()
    q = cases.fields(system, nvar=3, seed=23)

    def setup(t):
        _gpu_setup(1)(t)
        t.lib.tioga_b200_set_test_bound_(C.byref(C.c_int(2)), C.byref(C.c_int(chunk)))

    ref = run_system(oracle_lib, system, q_blocks=q, nvar=3)
    gpu = run_system(tb.library_path(), system, q_blocks=q, nvar=3, setup=setup)
    problems = diff_runs(system, ref, gpu)
    assert not problems, "\n".join(problems)


def _reduce(t):
    t.lib.tioga_reduce_fringes_()


@pytest.mark.parametrize("name,nfringe", [("cfg0", 1), ("cfg0", 3), ("cfg1-small-seed3", 2)])
def test_reduce_fringes_matches_oracle(name, nfringe, oracle_lib):
    """tioga_reduce_fringes_ after connectivity: iblanks (deep receptors become
    holes), surviving donor lists and the data update, against the oracle."""
    system = CASES[name]()
    q = cases.fields(system, nvar=5, seed=31)
    ref = run_system(oracle_lib, system, q_blocks=q, nfringe=nfringe, after=_reduce)
    gpu = run_system(tb.library_path(), system, q_blocks=q, nfringe=nfringe, setup=_gpu_setup(1), after=_reduce)
    problems = diff_runs(system, ref, gpu)
    assert not problems, "\n".join(problems)


def test_connectivity_after_reduce_fringes(oracle_lib):
    """A connectivity call after tioga_reduce_fringes_ (the shells moved in
    between) equals a fresh run: the holes the reduction made are undone."""
    import copy
    import ctypes as C
    from tioga_b200.capi import TiogaLibrary
    system = cases.config0(0)
    moved = copy.deepcopy(system)
    moved.blocks[1].x[:] = moved.blocks[1].x + np.array([0.031, -0.017, 0.022])
    t = TiogaLibrary(tb.library_path())
    t.init()
    t.register_system(copy.deepcopy(system))
    t.setnfringe(3)
    t.preprocess_grids()
    t.performconnectivity()
    t.lib.tioga_reduce_fringes_()
    for b in moved.blocks:
        t.blocks[b.tag]["x"][:] = b.x.reshape(-1)
    t.preprocess_grids()
    t.performconnectivity()
    got = {"iblank": {b.tag: t.iblank(b.tag).copy() for b in moved.blocks},
           "donors": {b.tag: t.getdonorinfo(b.tag) for b in moved.blocks}, "q": {}}
    cells = {}
    for b in moved.blocks:
        c = np.zeros(b.ncells, np.int32)
        t.lib.tioga_b200_getcelliblank_(C.byref(C.c_int(b.tag)), c.ctypes.data_as(C.c_void_p))
        cells[b.tag] = c
    t.delete()
    ref = run_system(oracle_lib, moved, nfringe=3)
    problems = diff_runs(moved, ref, got)
    assert not problems, "\n".join(problems)
    # cell iblanks of the new call, from its node iblanks (getCellIblanks,
    # highOrder.C:88-150): nothing left over from the reduction
    for b in moved.blocks:
        ib = got["iblank"][b.tag]
        want = []
        for nv, conn in b.cells:
            v = ib[conn]
            want.append(np.where((v == 0).any(axis=1), 0, np.where((v == -1).all(axis=1), -1, 1)))
        np.testing.assert_array_equal(cells[b.tag], np.concatenate(want))


@pytest.mark.parametrize("itype", ["row", "column"])
def test_writeoutputfiles_match_reference(itype, tmp_path, monkeypatch):
    """tioga_writeoutputfiles_ after the data update: the same flow files, byte
    for byte, as the compiled reference writes (tioga.C:526-531,
    MeshBlock.C:510-635)."""
    import os
    from tioga_b200.capi import TiogaLibrary
    from tests.conftest import REF_LIB
    if not os.path.exists(REF_LIB):
        pytest.skip("the compiled reference is not built here")
    system = cases.small_config1(1)
    q = cases.fields(system, nvar=3, seed=41)
    if itype == "column":
        q = [a.reshape(-1, 3).T.copy().reshape(-1) for a in q]
    files = {}
    for name, path in (("ref", REF_LIB), ("gpu", tb.library_path())):
        d = tmp_path / name
        d.mkdir()
        monkeypatch.chdir(d)
        t = TiogaLibrary(path)
        t.init()
        t.register_system(system)
        t.preprocess_grids()
        t.performconnectivity()
        qs = [a.copy() for a in q]
        for b, a in zip(system.blocks, qs):
            t.registersolution(b.tag, a)
        t.dataupdate_mb(3, itype)
        s = C.create_string_buffer(itype.encode())
        t.lib.tioga_writeoutputfiles_(C.byref(C.c_int(3)), s)
        t.delete()
        files[name] = {p.name: p.read_bytes() for p in sorted(d.iterdir())}
    assert sorted(files["gpu"]) == sorted(files["ref"]) == [f"flow{i:05d}.dat" for i in range(len(system.blocks))]
    for f in files["ref"]:
        assert files["gpu"][f] == files["ref"][f], f
