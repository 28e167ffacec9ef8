"""ctypes mirror of TIOGA's C API (src/tiogaInterface.C:36-328).

``TiogaLibrary`` binds any shared library that exports the TIOGA symbols:
this package's GPU library, the C restatement in ``oracle/`` or the compiled
reference.  The call sequence a solver makes is the reference's own:

    init -> registergrid_data_mb (per block) -> preprocess_grids ->
    performconnectivity -> registersolution (per block) -> dataupdate_mb

Scalars are passed by pointer and connectivity is 1-based, exactly as TIOGA
expects; ``registergrid_data_mb`` forwards its cell types as the trailing
varargs triples ``(int *nv, int *nc, int *vconn)``.  The library keeps the
caller's pointers (src/MeshBlock.C:37-72), so this class owns the arrays for
as long as the library may read them.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_P = C.c_void_p


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_P)


def _iref(v: int):
    return C.byref(C.c_int(int(v)))


class TiogaLibrary:
    """One loaded TIOGA-ABI library with its registered system."""

    def __init__(self, path: str):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.path = path
        self.lib = C.CDLL(path, mode=C.RTLD_LOCAL)
        self._keep = []          # arrays the library points into
        self.blocks = {}         # tag -> dict of host arrays
        self._order = []         # tags in registration order

    # -- lifecycle ---------------------------------------------------------
    def init(self):
        self.lib.tioga_init_.argtypes = [C.c_int]
        self.lib.tioga_init_.restype = None
        self.lib.tioga_init_(C.c_int(91))

    def delete(self):
        self.lib.tioga_delete_()
        self._keep.clear()
        self.blocks.clear()
        self._order.clear()

    # -- registration ------------------------------------------------------
    def registergrid_data_mb(self, bid: int, block, ibl=None, cell_gid=None, node_gid=None):
        """Register one cases.Block under block id ``bid`` (1-based).  ``ibl``
        may supply the iblank array (e.g. pinned host memory); ``cell_gid``
        the cells' uint64 global ids (tioga_b200_registercellgid_ here; the
        compiled reference takes them through its C++ class, by the test shim
        refshim_registergrid_gid_)."""
        x = np.ascontiguousarray(block.x, dtype=np.float64).reshape(-1)
        if ibl is None:
            ibl = np.ones(block.nnodes, dtype=np.int32)
        wbc = np.ascontiguousarray(block.wbc, dtype=np.int32) + 1
        obc = np.ascontiguousarray(block.obc, dtype=np.int32) + 1
        conns = []
        args = []
        for nv, conn in block.cells:
            c1 = np.ascontiguousarray(conn, dtype=np.int32).reshape(-1) + 1
            conns.append(c1)
            nvc = C.c_int(int(nv))
            ncc = C.c_int(int(conn.shape[0]))
            self._keep += [nvc, ncc]
            args += [C.byref(nvc), C.byref(ncc), _ptr(c1)]
        self._keep += [x, ibl, wbc, obc] + conns
        cbid, ctag, cnn = C.c_int(bid), C.c_int(block.tag), C.c_int(block.nnodes)
        cnw, cno, cnt = C.c_int(len(wbc)), C.c_int(len(obc)), C.c_int(len(block.cells))
        self._keep += [cbid, ctag, cnn, cnw, cno, cnt]
        regargs = (C.byref(cbid), C.byref(ctag), C.byref(cnn), _ptr(x), _ptr(ibl),
                   C.byref(cnw), C.byref(cno), _ptr(wbc), _ptr(obc), C.byref(cnt), *args)
        gid = None
        if cell_gid is not None:
            gid = np.ascontiguousarray(cell_gid, dtype=np.uint64)
            assert gid.shape == (block.ncells,)
            self._keep.append(gid)
        ngid = None
        if node_gid is not None:
            ngid = np.ascontiguousarray(node_gid, dtype=np.uint64)
            assert ngid.shape == (block.nnodes,)
            self._keep.append(ngid)
        if ngid is not None and hasattr(self.lib, "refshim_registergrid_gids_"):
            self.lib.refshim_registergrid_gids_(None if gid is None else _ptr(gid), _ptr(ngid), *regargs)
        elif gid is not None and hasattr(self.lib, "refshim_registergrid_gid_"):
            self.lib.refshim_registergrid_gid_(_ptr(gid), *regargs)
        else:
            self.lib.tioga_registergrid_data_mb_(*regargs)
            if gid is not None:
                self.lib.tioga_b200_registercellgid_(C.byref(ctag), _ptr(gid))
            if ngid is not None:
                if hasattr(self.lib, "tioga_oracle_set_node_gid"):
                    self.lib.tioga_oracle_set_node_gid(C.c_int(block.tag), _ptr(ngid))
                else:
                    self.lib.tioga_b200_registernodegid_(C.byref(ctag), _ptr(ngid))
        self.blocks[block.tag] = {"x": x, "iblank": ibl, "nnodes": block.nnodes,
                                  "ncells": block.ncells, "bid": bid}
        if block.tag not in self._order:
            self._order.append(block.tag)

    def registergrid_sys(self, sys: int, bid: int, block):
        """Register one cases.Block as block ``bid`` of overset system ``sys``
        (tioga_b200_registergrid_sys_, the batched form)."""
        x = np.ascontiguousarray(block.x, dtype=np.float64).reshape(-1)
        ibl = np.ones(block.nnodes, dtype=np.int32)
        wbc = np.ascontiguousarray(block.wbc, dtype=np.int32) + 1
        obc = np.ascontiguousarray(block.obc, dtype=np.int32) + 1
        args = []
        for nv, conn in block.cells:
            c1 = np.ascontiguousarray(conn, dtype=np.int32).reshape(-1) + 1
            nvc, ncc = C.c_int(int(nv)), C.c_int(int(conn.shape[0]))
            self._keep += [nvc, ncc, c1]
            args += [C.byref(nvc), C.byref(ncc), _ptr(c1)]
        scalars = [C.c_int(sys), C.c_int(block.tag), C.c_int(block.nnodes), C.c_int(len(wbc)),
                   C.c_int(len(obc)), C.c_int(len(block.cells))]
        self._keep += [x, ibl, wbc, obc] + scalars
        cs, ct, cn, cw, co, cty = scalars
        self.lib.tioga_b200_registergrid_sys_(
            C.byref(cs), C.byref(ct), C.byref(cn), _ptr(x), _ptr(ibl), C.byref(cw), C.byref(co), _ptr(wbc),
            _ptr(obc), C.byref(cty), *args)
        self.blocks[(sys, block.tag)] = {"x": x, "iblank": ibl, "nnodes": block.nnodes,
                                         "ncells": block.ncells, "bid": bid}

    def register_batch(self, systems):
        """Every system of a batch, system k under id k."""
        for k, system in enumerate(systems):
            for bid, b in enumerate(system.blocks, start=1):
                self.registergrid_sys(k, bid, b)

    def select_system(self, sys: int):
        self.lib.tioga_b200_select_system_(_iref(sys))

    def register_system(self, system, iblanks=None, cell_gids=None, node_gids=None):
        for bid, b in enumerate(system.blocks, start=1):
            self.registergrid_data_mb(bid, b, None if iblanks is None else iblanks[bid - 1],
                                      None if cell_gids is None else cell_gids[bid - 1],
                                      None if node_gids is None else node_gids[bid - 1])

    # -- settings ----------------------------------------------------------
    def setsymmetry(self, isym: int):
        self.lib.tioga_setsymmetry_(_iref(isym))

    def setnfringe(self, nfringe: int):
        self.lib.tioga_setnfringe_(_iref(nfringe))

    def setmexclude(self, mexclude: int):
        self.lib.tioga_setmexclude_(_iref(mexclude))

    def setresolutions_multi(self, tag: int, nres: np.ndarray, cres: np.ndarray):
        nres = np.ascontiguousarray(nres, dtype=np.float64)
        cres = np.ascontiguousarray(cres, dtype=np.float64)
        self._keep += [nres, cres]
        self.lib.tioga_setresolutions_multi_(_iref(tag), _ptr(nres), _ptr(cres))

    # -- the hot path ------------------------------------------------------
    def preprocess_grids(self):
        self.lib.tioga_preprocess_grids_()

    def performconnectivity(self):
        self.lib.tioga_performconnectivity_()

    def registersolution(self, tag: int, q: np.ndarray):
        assert q.dtype == np.float64 and q.flags.c_contiguous
        self._keep.append(q)
        self.lib.tioga_registersolution_(_iref(tag), _ptr(q))

    def dataupdate_mb(self, nvar: int, itype: str = "row"):
        s = C.create_string_buffer(itype.encode())
        self.lib.tioga_dataupdate_mb_(_iref(nvar), s)

    # -- queries -----------------------------------------------------------
    def getdonorcount(self, tag: int):
        d, f = C.c_int(0), C.c_int(0)
        self.lib.tioga_getdonorcount_(_iref(tag), C.byref(d), C.byref(f))
        return d.value, f.value

    def getdonorinfo(self, tag: int):
        """Returns (receptors (dcount,4), indices (fcount,), frac (fcount,))."""
        d, f = self.getdonorcount(tag)
        rec = np.zeros(4 * max(d, 1), dtype=np.int32)
        ind = np.zeros(max(f, 1), dtype=np.int32)
        frac = np.zeros(max(f, 1), dtype=np.float64)
        dc = C.c_int(d)
        if d > 0:
            self.lib.tioga_getdonorinfo_(_iref(tag), _ptr(rec), _ptr(ind), _ptr(frac), C.byref(dc))
        return rec[:4 * d].reshape(d, 4), ind[:f], frac[:f]

    def getreceptorinfo(self) -> np.ndarray:
        """tioga::getReceptorInfo: (n, 4) int32 rows of (receptor node,
        receptor mesh tag, donor cell global id low word, high word)."""
        if hasattr(self.lib, "refshim_getreceptorinfo_"):
            self.lib.refshim_getreceptorinfo_.restype = C.c_int
            n = self.lib.refshim_getreceptorinfo_(None, C.c_int(0))
            out = np.zeros(max(n, 1), dtype=np.int32)
            self.lib.refshim_getreceptorinfo_(_ptr(out), C.c_int(n))
            return out[:n].reshape(-1, 4)
        nr = C.c_int(0)
        self.lib.tioga_b200_getreceptorcount_(C.byref(nr))
        out = np.zeros(max(4 * nr.value, 1), dtype=np.int32)
        if nr.value > 0:
            self.lib.tioga_b200_getreceptorinfo_(_ptr(out))
        return out[:4 * nr.value].reshape(-1, 4)

    def iblank(self, tag: int) -> np.ndarray:
        return self.blocks[tag]["iblank"]

    @property
    def tags(self):
        return list(self._order)


def run_system(lib_path: str, system, q_blocks=None, nvar: int = 5, itype: str = "row",
               isym=None, nfringe=None, mexclude=None, resolutions=None, setup=None, after=None,
               cell_gids=None, node_gids=None):
    """Drive one library through the full TIOGA call sequence and collect
    every observable: iblank per block, donor info per block and the updated
    fields.  ``q_blocks`` are copied (the library updates them in place).
    With ``cell_gids`` (per block, uint64 per cell) the blocks carry cell
    global ids and ``out["receptorinfo"]`` is getReceptorInfo's result; with
    ``node_gids`` (per block, uint64 per node) the blocks carry node global
    ids (the node-GID merge of coincident query points uses them)."""
    t = TiogaLibrary(lib_path)
    t.init()
    t.register_system(system, cell_gids=cell_gids, node_gids=node_gids)
    if isym is not None:
        t.setsymmetry(isym)
    if nfringe is not None:
        t.setnfringe(nfringe)
    if mexclude is not None:
        t.setmexclude(mexclude)
    if resolutions is not None:
        for tag, (nres, cres) in resolutions.items():
            t.setresolutions_multi(tag, nres, cres)
    if setup is not None:
        setup(t)
    t.preprocess_grids()
    t.performconnectivity()
    out = {"iblank": {}, "donors": {}, "q": {}}
    if after is not None:
        out["after"] = after(t)
    for b in system.blocks:
        out["iblank"][b.tag] = t.iblank(b.tag).copy()
        out["donors"][b.tag] = t.getdonorinfo(b.tag)
    if cell_gids is not None:
        out["receptorinfo"] = t.getreceptorinfo()
    if q_blocks is not None:
        qs = [np.array(q, dtype=np.float64, copy=True) for q in q_blocks]
        for b, q in zip(system.blocks, qs):
            t.registersolution(b.tag, q)
        t.dataupdate_mb(nvar, itype)
        for b, q in zip(system.blocks, qs):
            out["q"][b.tag] = q
    t.delete()
    return out


def run_batch(lib_path: str, systems, q_sets=None, nvar: int = 5, itype: str = "row", setup=None):
    """The batched form: every system registered in one instance
    (tioga_b200_registergrid_sys_), one preprocess, one connectivity and one
    data update for all of them.  Returns one result per system in the
    layout of ``run_system``."""
    t = TiogaLibrary(lib_path)
    t.init()
    t.register_batch(systems)
    if setup is not None:
        setup(t)
    t.preprocess_grids()
    t.performconnectivity()
    outs = []
    for k, system in enumerate(systems):
        t.select_system(k)
        out = {"iblank": {}, "donors": {}, "q": {}}
        for b in system.blocks:
            out["iblank"][b.tag] = t.blocks[(k, b.tag)]["iblank"].copy()
            out["donors"][b.tag] = t.getdonorinfo(b.tag)
        outs.append(out)
    if q_sets is not None:
        qs = []
        for k, system in enumerate(systems):
            t.select_system(k)
            qk = [np.array(q, dtype=np.float64, copy=True) for q in q_sets[k]]
            for b, q in zip(system.blocks, qk):
                t.registersolution(b.tag, q)
            qs.append(qk)
        t.dataupdate_mb(nvar, itype)
        for k, system in enumerate(systems):
            for b, q in zip(system.blocks, qs[k]):
                outs[k]["q"][b.tag] = q
    t.delete()
    return outs
