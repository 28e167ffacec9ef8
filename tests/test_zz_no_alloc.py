"""The allocation-free interpolation entry point (tioga_b200_interpolate_noalloc_).

It serves callers that cannot allocate device memory while they update their
fields -- a solver stepping inside a captured CUDA graph, or one whose memory
pool must not see cudaMalloc's device-wide synchronisation.  Checked through
the C ABI against the regular data update (tioga_dataupdate_mb_) on the same
connectivity, bit for bit, on two updates in a row in the row and the column
layouts, and on a third captured in a CUDA graph and replayed; the staging array is
shared by all calls, so the second call also shows that nothing is left over
from the first.  The file name sorts last so a stop-at-first-failure run has
run every other test before this one.
"""
import ctypes as C

import numpy as np
import pytest

import tioga_b200 as tb
from tioga_b200 import cases
from tioga_b200.capi import TiogaLibrary

pytestmark = pytest.mark.gpu

NOALLOC_MAX_VALUES = 1 << 20


def _stencils(t, system, offsets):
    """Donor stencils of every block in the flat node numbering (row layout)."""
    inode, w, nw, recv = [], [], [], []
    for b in system.blocks:
        rec, ind, frac = t.getdonorinfo(b.tag)
        k = 0
        for i in range(rec.shape[0]):
            n = int(rec[i, 3])
            row_i = np.zeros(9, np.int32)
            row_w = np.zeros(9, np.float64)
            row_i[:n] = offsets[b.tag] + ind[k:k + n]
            row_w[:n] = frac[k:k + n]
            inode.append(row_i)
            w.append(row_w)
            nw.append(n)
            recv.append(offsets[system.blocks[rec[i, 2]].tag] + rec[i, 1])
            k += n + 1
    return (np.array(inode, np.int32).reshape(-1), np.array(w).reshape(-1),
            np.array(nw, np.int32), np.array(recv, np.int32))


def test_noalloc_matches_dataupdate_twice():
    import torch
    system = cases.small_config1(1)
    nvar = 5
    q0 = cases.fields(system, nvar=nvar, seed=21)
    t = TiogaLibrary(tb.library_path())
    lib = tb.extras(t.lib)
    fn = lib.tioga_b200_interpolate_noalloc_
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_longlong,
                   C.c_int, C.c_int, C.c_void_p]
    t.init()
    t.register_system(system)
    t.preprocess_grids()
    t.performconnectivity()
    assert lib.tioga_b200_last_error() == 0
    # the regular entry point, twice in a row on host arrays
    qs = [np.array(q, copy=True) for q in q0]
    for b, q in zip(system.blocks, qs):
        t.registersolution(b.tag, q)
    t.dataupdate_mb(nvar, "row")
    first = np.concatenate([q.copy() for q in qs])
    t.dataupdate_mb(nvar, "row")
    second = np.concatenate([q.copy() for q in qs])
    # the allocation-free entry point on the same stencils, flat row layout
    offsets, off = {}, 0
    for b in system.blocks:
        offsets[b.tag] = off
        off += b.nnodes
    inode, w, nw, recv = _stencils(t, system, offsets)
    nrec = int(nw.shape[0])
    assert nrec > 0
    dev = torch.device("cuda:0")
    d_inode = torch.from_numpy(inode).to(dev)
    d_w = torch.from_numpy(w).to(dev)
    d_nw = torch.from_numpy(nw).to(dev)
    d_recv = torch.from_numpy(recv).to(dev)
    d_q = torch.from_numpy(np.concatenate(q0)).to(dev)
    stream = torch.cuda.current_stream().cuda_stream
    for expect in (first, second):
        rc = fn(d_inode.data_ptr(), d_w.data_ptr(), d_nw.data_ptr(), d_recv.data_ptr(), nrec,
                d_q.data_ptr(), off, nvar, 0, stream)
        assert rc == 0
        torch.cuda.synchronize()
        got = d_q.cpu().numpy()
        assert np.array_equal(got.view(np.int64), expect.view(np.int64))
    # inside a captured CUDA graph, the case the entry point exists for: a
    # third update, captured once (after the eager calls above made the
    # first-call set-up) and replayed, against the regular entry point's
    t.dataupdate_mb(nvar, "row")
    third = np.concatenate([q.copy() for q in qs])
    graph = torch.cuda.CUDAGraph()
    rcs = []
    with torch.cuda.graph(graph):
        rcs.append(fn(d_inode.data_ptr(), d_w.data_ptr(), d_nw.data_ptr(), d_recv.data_ptr(), nrec,
                      d_q.data_ptr(), off, nvar, 0, torch.cuda.current_stream().cuda_stream))
    assert rcs == [0]
    torch.cuda.synchronize()
    assert np.array_equal(d_q.cpu().numpy().view(np.int64), second.view(np.int64))  # captured, not run
    graph.replay()
    torch.cuda.synchronize()
    assert np.array_equal(d_q.cpu().numpy().view(np.int64), third.view(np.int64))
    # the column layout (q[k*nnodes+node]) against tioga_dataupdate_mb_'s, twice
    qc = [np.array(q, copy=True) for q in q0]  # read as column-layout arrays of each block
    for b, q in zip(system.blocks, qc):
        t.registersolution(b.tag, q)
    expect_col = []
    for _ in range(2):
        t.dataupdate_mb(nvar, "column")
        flat = np.zeros(off * nvar)
        for b, q in zip(system.blocks, qc):
            for k in range(nvar):
                flat[k * off + offsets[b.tag]:k * off + offsets[b.tag] + b.nnodes] = q[k * b.nnodes:(k + 1) * b.nnodes]
        expect_col.append(flat)
    flat0 = np.zeros(off * nvar)
    for b, q in zip(system.blocks, q0):
        for k in range(nvar):
            flat0[k * off + offsets[b.tag]:k * off + offsets[b.tag] + b.nnodes] = q[k * b.nnodes:(k + 1) * b.nnodes]
    d_qc = torch.from_numpy(flat0).to(dev)
    for expect in expect_col:
        rc = fn(d_inode.data_ptr(), d_w.data_ptr(), d_nw.data_ptr(), d_recv.data_ptr(), nrec,
                d_qc.data_ptr(), off, nvar, 1, stream)
        assert rc == 0
        torch.cuda.synchronize()
        assert np.array_equal(d_qc.cpu().numpy().view(np.int64), expect.view(np.int64))
    # sizes beyond the fixed staging array are refused and leave q untouched
    before = d_q.cpu().numpy().copy()
    big = NOALLOC_MAX_VALUES // nvar + 1
    rc = fn(d_inode.data_ptr(), d_w.data_ptr(), d_nw.data_ptr(), d_recv.data_ptr(), big,
            d_q.data_ptr(), off, nvar, 0, stream)
    assert rc == -1
    torch.cuda.synchronize()
    assert np.array_equal(d_q.cpu().numpy(), before)
    t.delete()
