"""Failure handling, injected on the host: bad caller inputs, device bounds
lowered until they run out, and serving requests that are refused, cancelled
or waited for with a time limit.  Every case must end in an error status the
host reads (tioga_b200_last_error(), a request status), with no crash and
with the library usable afterwards -- the next good call must equal the
oracle.  The reference's counterpart is its abort on a weight outside
[-0.2, 1.2] (src/bookKeeping.C:521-529); this library reports instead.
Nothing here faults the GPU: each bad input is refused before a kernel can
index with it, and each lowered bound is a counted loop that gives up."""
import ctypes as C

import numpy as np
import pytest

import tioga_b200 as tb
from tioga_b200 import cases
from tioga_b200.capi import TiogaLibrary, run_system
from tests.compare import diff_runs

pytestmark = pytest.mark.gpu

ERR_CAPACITY = 1 << 1
ERR_FLOOD_FILL = 1 << 3


def _lib():
    t = TiogaLibrary(tb.library_path())
    tb.extras(t.lib)
    return t


def _run_after(t, system):
    """The rest of run_system's sequence on an instance that is registered."""
    t.preprocess_grids()
    t.performconnectivity()
    out = {"iblank": {}, "donors": {}, "q": {}}
    for b in system.blocks:
        out["iblank"][b.tag] = t.iblank(b.tag).copy()
        out["donors"][b.tag] = t.getdonorinfo(b.tag)
    return out


def test_unsupported_cell_type_is_refused():
    system = cases.small_config0(0)
    t = _lib()
    t.init()
    b = system.blocks[0]
    nv, conn = b.cells[0]
    bad = cases.Block(b.tag, b.x, [(7, np.zeros((conn.shape[0], 7), np.int32))], b.wbc, b.obc)
    t.registergrid_data_mb(1, bad)
    assert t.lib.tioga_b200_last_error() != 0
    t.delete()


def test_connectivity_index_out_of_range_then_recovers(oracle_lib):
    system = cases.small_config0(0)
    sh = system.blocks[1]
    nv, conn = sh.cells[0]
    conn_bad = conn.copy()
    conn_bad[5, 3] = sh.nnodes + 3  # past the block's nodes (0-based here, +1 in the ABI)
    bad = cases.Block(sh.tag, sh.x, [(nv, conn_bad)], sh.wbc, sh.obc)
    t = _lib()
    t.init()
    t.registergrid_data_mb(1, system.blocks[0])
    t.registergrid_data_mb(2, bad)
    t.preprocess_grids()
    assert t.lib.tioga_b200_last_error() != 0
    t.performconnectivity()  # refused: no preprocessed topology
    assert t.lib.tioga_b200_last_error() != 0
    # the same instance with the block registered again, correctly
    t.registergrid_data_mb(2, sh)
    gpu = _run_after(t, system)
    assert t.lib.tioga_b200_last_error() == 0
    t.delete()
    ref = run_system(oracle_lib, system)
    assert not diff_runs(system, ref, gpu, exact_q=False)


def test_wall_node_out_of_range_is_refused():
    system = cases.small_config0(0)
    sh = system.blocks[1]
    wbc = sh.wbc.copy()
    wbc[0] = -7
    bad = cases.Block(sh.tag, sh.x, sh.cells, wbc, sh.obc)
    t = _lib()
    t.init()
    t.registergrid_data_mb(1, system.blocks[0])
    t.registergrid_data_mb(2, bad)
    t.preprocess_grids()
    assert t.lib.tioga_b200_last_error() != 0
    t.delete()


def test_nan_coordinate_then_recovers(oracle_lib):
    system = cases.small_config1(1)
    t = _lib()
    t.init()
    t.register_system(system)
    x = t.blocks[system.blocks[1].tag]["x"]  # the array the library reads
    keep = x[40]
    x[40] = np.nan
    t.preprocess_grids()
    assert t.lib.tioga_b200_last_error() != 0
    x[40] = keep
    t.preprocess_grids()
    assert t.lib.tioga_b200_last_error() == 0
    keep41 = x[41]
    x[41] = np.inf  # a node moved to infinity before a connectivity call
    t.performconnectivity()
    assert t.lib.tioga_b200_last_error() != 0
    x[41] = keep41
    t.performconnectivity()
    assert t.lib.tioga_b200_last_error() == 0
    gpu = {"iblank": {b.tag: t.iblank(b.tag).copy() for b in system.blocks},
           "donors": {b.tag: t.getdonorinfo(b.tag) for b in system.blocks}, "q": {}}
    t.delete()
    ref = run_system(oracle_lib, system)
    assert not diff_runs(system, ref, gpu, exact_q=False)


@pytest.mark.parametrize("which,value,bit", [(0, 1, ERR_FLOOD_FILL), (1, 1, ERR_CAPACITY)])
def test_lowered_device_bound_reports_then_recovers(oracle_lib, which, value, bit):
    """A hole-map fill allowed one round, a donor-record list of one entry:
    the kernels give up at the bound, set their error bit, and the host
    reports it; with the bound restored the next call is exact again."""
    system = cases.small_config1(1)
    t = _lib()
    t.init()
    t.register_system(system)
    t.preprocess_grids()
    tb.set_int(t.lib, "tioga_b200_set_precision_", 1)
    t.lib.tioga_b200_set_test_bound_(C.byref(C.c_int(which)), C.byref(C.c_int(value)))
    t.performconnectivity()
    err = t.lib.tioga_b200_last_error()
    assert err & bit, err
    assert tb.stats(t.lib)["error"] & bit
    t.lib.tioga_b200_set_test_bound_(C.byref(C.c_int(which)), C.byref(C.c_int(0)))
    t.performconnectivity()
    assert t.lib.tioga_b200_last_error() == 0
    gpu = {"iblank": {b.tag: t.iblank(b.tag).copy() for b in system.blocks},
           "donors": {b.tag: t.getdonorinfo(b.tag) for b in system.blocks}, "q": {}}
    t.delete()
    ref = run_system(oracle_lib, system)
    assert not diff_runs(system, ref, gpu, exact_q=False)


def _server_systems():
    return cases.small_config2(2, nsys=3)


def test_server_refuses_a_system_over_the_budget():
    from tioga_b200.serving import Server
    systems = _server_systems()
    srv = Server(budget_bytes=1 << 20, nslots=2)  # 1 MiB: no system fits
    srv.add_system(0, systems[0])
    r = srv.wait(srv.submit(0))
    assert r["rc"] == Server.OVER_BUDGET
    srv.close()


def test_server_cancel_and_bounded_wait():
    from tioga_b200.serving import Server
    systems = _server_systems()
    srv = Server(budget_bytes=8 << 30, nslots=1)
    srv.add_system(0, systems[0])
    # requests of one system run one at a time in order: the later ones queue
    tickets = [srv.submit(0) for _ in range(4)]
    assert srv.wait(tickets[3], timeout_ms=0.0)["rc"] == Server.TIMED_OUT
    assert srv.cancel(tickets[3])
    results = [srv.wait(t) for t in tickets[:3]]
    assert all(r["rc"] == 0 for r in results)
    assert srv.wait(tickets[3])["rc"] == Server.CANCELLED
    assert not srv.cancel(tickets[0])  # finished and collected
    srv.close()
