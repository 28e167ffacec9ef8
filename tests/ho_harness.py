"""Drives the high-order path (tioga_performconnectivity_highorder_ and the
point data update, src/tioga.C:162-178, src/highOrder.C) for the tests.

For the oracle and the compiled reference, the element arithmetic comes from
the Lagrange-hex callbacks in oracle/_ref/libho_callbacks.so, passed to
tioga_set_highorder_callback_ as C function pointers.  The callbacks receive
no block id; the oracle names the block through its block hook, the compiled
reference runs in a configuration where receptor-side calls only concern one
block and donor-side calls another (`roles`).  The GPU library gets the same
element description natively (tioga_b200_set_highorder_lagrange_)."""
import ctypes as C
import os

import numpy as np

from tioga_b200.capi import TiogaLibrary

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CB_LIB = os.path.join(ROOT, "oracle", "_ref", "libho_callbacks.so")


def run_highorder(lib_path, system, ho, nvar, q_dof, mode, resolutions=None, setup=None):
    """mode: "hook" (oracle), "roles" (compiled reference: receptor block
    index 1, donor block index 0) or "gpu".  Returns iblanks, cell iblanks
    (oracle and GPU), point donors (oracle and GPU) and the updated DOF
    arrays."""
    t = TiogaLibrary(lib_path)
    t.init()
    t.register_system(system)
    if resolutions is not None:
        for tag, (nres, cres) in resolutions.items():
            t.setresolutions_multi(tag, nres, cres)
    keep = []
    if mode in ("hook", "roles"):
        cb = C.CDLL(CB_LIB)
        for ib, h in enumerate(ho):
            xd = np.ascontiguousarray(h.xdof, dtype=np.float64)
            keep.append(xd)
            cb.ho_register(C.c_int(ib), C.c_int(h.p), C.c_int(xd.shape[0]), xd.ctypes.data_as(C.c_void_p))
        cb.ho_set_nvar(C.c_int(nvar))
        if mode == "hook":
            cb.ho_set_roles(C.c_int(-1), C.c_int(-1))
            t.lib.tioga_oracle_set_block_hook.argtypes = [C.c_void_p]
            t.lib.tioga_oracle_set_block_hook(C.cast(cb.ho_set_block, C.c_void_p))
        else:
            cb.ho_set_roles(C.c_int(1), C.c_int(0))
        fns = [C.cast(getattr(cb, n), C.c_void_p) for n in
               ("ho_nodes_per_cell", "ho_receptor_nodes", "ho_inclusion", "ho_frac", "ho_to_modal")]
        t.lib.tioga_set_highorder_callback_.argtypes = [C.c_void_p] * 5
        t.lib.tioga_set_highorder_callback_(*fns)
    else:
        for b, h in zip(system.blocks, ho):
            xd = np.ascontiguousarray(h.xdof, dtype=np.float64)
            keep.append(xd)
            t.lib.tioga_b200_set_highorder_lagrange_(C.byref(C.c_int(b.tag)), C.byref(C.c_int(h.p)),
                                                     xd.ctypes.data_as(C.c_void_p))
    if setup is not None:
        setup(t)
    t.preprocess_grids()
    t.performconnectivity()
    t.lib.tioga_performconnectivity_highorder_()
    out = {"iblank": {}, "cells": {}, "points": {}, "q": {}}
    for b in system.blocks:
        out["iblank"][b.tag] = t.iblank(b.tag).copy()
    if mode == "hook":
        for ib, b in enumerate(system.blocks):
            n = t.lib.tioga_oracle_pointdonors(C.c_int(b.tag), None, None)
            rec = np.zeros((max(n, 1), 4), np.int32)
            w = np.zeros((max(n, 1), 1331), np.float64)
            t.lib.tioga_oracle_pointdonors(C.c_int(b.tag), rec.ctypes.data_as(C.c_void_p),
                                           w.ctypes.data_as(C.c_void_p))
            # the callbacks report the donor cell's first value (1-based); as a cell id
            npts = (ho[ib].p + 1) ** 3
            rec[:n, 2] = (rec[:n, 2] - 1) // (npts * nvar)
            out["points"][b.tag] = (rec[:n], w[:n])
    elif mode == "gpu":
        st = (C.c_longlong * 8)()
        t.lib.tioga_b200_highorder_stats_(st)
        out["stats"] = list(st)
        for b in system.blocks:
            n = t.lib.tioga_b200_pointdonors_(C.byref(C.c_int(b.tag)), None, None)
            rec = np.zeros((max(n, 1), 4), np.int32)
            w = np.zeros((max(n, 1), 1331), np.float64)
            t.lib.tioga_b200_pointdonors_(C.byref(C.c_int(b.tag)), rec.ctypes.data_as(C.c_void_p),
                                          w.ctypes.data_as(C.c_void_p))
            out["points"][b.tag] = (rec[:n], w[:n])
    qs = [np.array(q, dtype=np.float64, copy=True) for q in q_dof]
    for b, q in zip(system.blocks, qs):
        t.registersolution(b.tag, q)
    t.dataupdate_mb(nvar, "row")
    for b, q in zip(system.blocks, qs):
        out["q"][b.tag] = q
    for b in system.blocks:  # after clearOrphans (the reference exposes none for every block)
        cell = np.zeros(b.ncells, np.int32)
        if mode == "hook":
            t.lib.tioga_oracle_getcelliblank(C.c_int(b.tag), cell.ctypes.data_as(C.c_void_p))
            out["cells"][b.tag] = cell
        elif mode == "gpu":
            t.lib.tioga_b200_getcelliblank_(C.byref(C.c_int(b.tag)), cell.ctypes.data_as(C.c_void_p))
            out["cells"][b.tag] = cell
    t.delete()
    del keep
    return out


def diff_highorder(system, a, b, points=True):
    """Mismatches between two high-order runs: iblanks, cell iblanks,
    point donors and weights, updated DOF values (bit for bit)."""
    out = []
    for blk in system.blocks:
        t = blk.tag
        if not np.array_equal(a["iblank"][t], b["iblank"][t]):
            out.append(f"tag {t}: iblank differs at {(a['iblank'][t] != b['iblank'][t]).sum()} nodes")
        if t in a["cells"] and t in b["cells"] and not np.array_equal(a["cells"][t], b["cells"][t]):
            out.append(f"tag {t}: cell iblank differs at {(a['cells'][t] != b['cells'][t]).sum()} cells")
        if points and t in a["points"] and t in b["points"]:
            ra, wa = a["points"][t]
            rb, wb = b["points"][t]
            if ra.shape != rb.shape or not np.array_equal(ra, rb):
                out.append(f"tag {t}: point donor records differ ({ra.shape[0]} vs {rb.shape[0]})")
            elif not np.array_equal(wa.view(np.int64), wb.view(np.int64)):
                out.append(f"tag {t}: point weights differ at {(wa != wb).sum()}, max {np.abs(wa - wb).max():.3e}")
        qa, qb = a["q"][t], b["q"][t]
        if not np.array_equal(qa.view(np.int64), qb.view(np.int64)):
            d = np.abs(qa - qb)
            out.append(f"tag {t}: DOF values differ at {(qa != qb).sum()}, max {d.max():.3e}")
    return out
