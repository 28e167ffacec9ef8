"""The serving form through its C ABI (tioga_b200_server_*): a request loop
over many resident overset systems, each request one time step of one system
(rigid motions of some blocks, then preprocess, connectivity and the data
update).  See include/tioga_b200.h for the scheduling and admission rules.

    srv = Server(budget_bytes=40 << 30, nslots=4)
    srv.add_system(0, system)                       # cases.System
    t = srv.submit(0, moves=[(2, A, b)], q=q_blocks, ibl_out=ibls)
    info = srv.wait(t)                              # latency, counts

The arrays handed over stay owned by this object (the library keeps their
pointers): each system's coordinates (written back by the library when the
system is evicted), iblank, boundary lists and connectivity.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import library_path

_P = C.c_void_p


def rigid(rng: np.random.Generator, centre, max_deg: float = 2.0, max_shift: float = 0.0):
    """A rigid motion as (A, b): a rotation by U(0, max_deg) degrees about a
    random axis through `centre`, then a translation of length
    U(0, max_shift) in a random direction."""
    ax = rng.normal(size=3)
    ax /= np.linalg.norm(ax)
    th = np.deg2rad(rng.uniform(0.0, max_deg))
    K = np.array([[0.0, -ax[2], ax[1]], [ax[2], 0.0, -ax[0]], [-ax[1], ax[0], 0.0]])
    A = np.eye(3) + np.sin(th) * K + (1.0 - np.cos(th)) * (K @ K)
    d = rng.normal(size=3)
    d *= rng.uniform(0.0, max_shift) / np.linalg.norm(d)
    c = np.asarray(centre, dtype=np.float64)
    return A, c - A @ c + d


def apply_rigid(x: np.ndarray, A: np.ndarray, b: np.ndarray) -> np.ndarray:
    """x <- A x + b evaluated as the device does, component k as
    ((A[k,0] x + A[k,1] y) + A[k,2] z) + b[k] (same bits)."""
    x0, x1, x2 = x[:, 0].copy(), x[:, 1].copy(), x[:, 2].copy()
    for k in range(3):
        x[:, k] = ((A[k, 0] * x0 + A[k, 1] * x1) + A[k, 2] * x2) + b[k]
    return x


class Server:
    def __init__(self, budget_bytes: int, nslots: int = 4, max_resident: int = 200, lib_path: str | None = None):
        self.lib = C.CDLL(lib_path or library_path(), mode=C.RTLD_LOCAL)
        L = self.lib
        L.tioga_b200_server_create.restype = _P
        L.tioga_b200_server_create.argtypes = [C.c_longlong, C.c_int, C.c_int]
        L.tioga_b200_server_destroy.argtypes = [_P]
        L.tioga_b200_server_add_block.restype = C.c_int
        L.tioga_b200_server_add_block.argtypes = [_P, C.c_int, C.c_int, C.c_int, _P, _P, C.c_int, C.c_int, _P, _P,
                                                  C.c_int, _P, _P, _P]
        L.tioga_b200_server_submit_fields.restype = C.c_longlong
        L.tioga_b200_server_submit_fields.argtypes = [_P, C.c_int, C.c_int, _P, _P, C.c_int, _P, C.c_int, _P]
        L.tioga_b200_server_wait.restype = C.c_int
        L.tioga_b200_server_wait.argtypes = [_P, C.c_longlong, _P, _P]
        L.tioga_b200_server_wait_timeout.restype = C.c_int
        L.tioga_b200_server_wait_timeout.argtypes = [_P, C.c_longlong, C.c_double, _P, _P]
        L.tioga_b200_server_cancel.restype = C.c_int
        L.tioga_b200_server_cancel.argtypes = [_P, C.c_longlong]
        L.tioga_b200_server_stats.argtypes = [_P, _P]
        self.h = L.tioga_b200_server_create(int(budget_bytes), int(nslots), int(max_resident))
        if not self.h:
            raise RuntimeError("tioga_b200_server_create failed (no CUDA device?)")
        self.systems = {}
        self._keep = {}      # ticket -> arrays of an in-flight request

    def add_system(self, sys_id: int, system, x_arrays=None, ibl_arrays=None):
        """Register every block of a cases.System as system `sys_id`.
        x_arrays / ibl_arrays may supply the (N, 3) float64 coordinate and
        int32 iblank arrays (e.g. pinned memory); by default copies are made."""
        blocks = []
        for i, b in enumerate(system.blocks):
            x = np.ascontiguousarray(b.x, dtype=np.float64).copy() if x_arrays is None else x_arrays[i]
            ibl = np.ones(b.nnodes, dtype=np.int32) if ibl_arrays is None else ibl_arrays[i]
            wbc = np.ascontiguousarray(b.wbc, dtype=np.int32) + 1
            obc = np.ascontiguousarray(b.obc, dtype=np.int32) + 1
            conns = [np.ascontiguousarray(conn, dtype=np.int32).reshape(-1) + 1 for _, conn in b.cells]
            nv = np.array([nv for nv, _ in b.cells], dtype=np.int32)
            nc = np.array([conn.shape[0] for _, conn in b.cells], dtype=np.int32)
            cptr = (_P * len(conns))(*[c.ctypes.data for c in conns])
            rc = self.lib.tioga_b200_server_add_block(
                self.h, int(sys_id), int(b.tag), int(b.nnodes), x.ctypes.data, ibl.ctypes.data, len(wbc), len(obc),
                wbc.ctypes.data, obc.ctypes.data, len(conns), nv.ctypes.data, nc.ctypes.data, C.cast(cptr, _P))
            if rc:
                raise RuntimeError(f"server_add_block failed for system {sys_id} tag {b.tag}")
            blocks.append({"tag": b.tag, "x": x, "ibl": ibl, "keep": (wbc, obc, conns, nv, nc, cptr),
                           "nnodes": b.nnodes})
        self.systems[sys_id] = blocks

    def submit(self, sys_id: int, moves=(), q=None, nvar: int = 5, ibl_out=None, q_device=None) -> int:
        """moves: [(tag, A (3, 3), b (3,))]; q: per-block ROW solutions
        (float64, nnodes*nvar, updated in place) or None; ibl_out: per-block
        int32 arrays for this request's iblank, or None.  q_device: per-block
        float64 CUDA tensors (or device pointers) instead of host q."""
        tags = np.array([m[0] for m in moves], dtype=np.int32)
        mv = np.zeros((max(len(moves), 1), 12), dtype=np.float64)
        for i, (_, A, b) in enumerate(moves):
            mv[i, :9] = np.asarray(A, dtype=np.float64).reshape(9)
            mv[i, 9:] = np.asarray(b, dtype=np.float64)
        keep = [tags, mv]
        qp = None
        if q_device is not None:
            ptrs = [a if isinstance(a, int) else a.data_ptr() for a in q_device]
            qp = (_P * len(ptrs))(*ptrs)
            keep += [qp, list(q_device)]
        elif q is not None:
            for a in q:
                assert a.dtype == np.float64 and a.flags.c_contiguous
            qp = (_P * len(q))(*[a.ctypes.data for a in q])
            keep += [qp, list(q)]
        ip = None
        if ibl_out is not None:
            for a in ibl_out:
                assert a.dtype == np.int32 and a.flags.c_contiguous
            ip = (_P * len(ibl_out))(*[a.ctypes.data for a in ibl_out])
            keep += [ip, list(ibl_out)]
        t = self.lib.tioga_b200_server_submit_fields(self.h, int(sys_id), len(moves), tags.ctypes.data,
                                                     mv.ctypes.data, int(nvar), None if qp is None else C.cast(qp, _P),
                                                     1 if q_device is not None else 0,
                                                     None if ip is None else C.cast(ip, _P))
        if t <= 0:
            raise RuntimeError(f"server_submit failed for system {sys_id}")
        self._keep[t] = keep
        return t

    # request statuses besides 0 and the engine's error codes
    OVER_BUDGET, CANCELLED, TIMED_OUT = -3, -4, -5

    def wait(self, ticket: int, timeout_ms: float | None = None) -> dict:
        """The request's result; with timeout_ms, rc == TIMED_OUT when it is
        not done by then (the ticket stays valid)."""
        times = (C.c_double * 6)()
        counts = (C.c_longlong * 4)()
        if timeout_ms is None:
            rc = self.lib.tioga_b200_server_wait(self.h, C.c_longlong(ticket), C.cast(times, _P),
                                                 C.cast(counts, _P))
        else:
            rc = self.lib.tioga_b200_server_wait_timeout(self.h, C.c_longlong(ticket), C.c_double(timeout_ms),
                                                         C.cast(times, _P), C.cast(counts, _P))
            if rc == self.TIMED_OUT:
                return {"rc": rc}
        self._keep.pop(ticket, None)
        return {"rc": rc, "latency_ms": times[0], "queue_ms": times[1], "service_ms": times[2],
                "preprocess_ms": times[3], "connectivity_ms": times[4], "dataupdate_ms": times[5],
                "nquery": counts[0], "nreceptor": counts[1], "nhole": counts[2]}

    def cancel(self, ticket: int) -> bool:
        """Cancel a request that has not started (it then completes with
        rc == CANCELLED); False when it runs or is done."""
        return self.lib.tioga_b200_server_cancel(self.h, C.c_longlong(ticket)) == 0

    def stats(self) -> dict:
        out = (C.c_longlong * 16)()
        self.lib.tioga_b200_server_stats(self.h, C.cast(out, _P))
        keys = ["resident", "bytes", "admissions", "evictions", "completed", "queued", "budget", "peak_bytes",
                "pool_reserved_at_create", "pool_bytes"]
        return {k: int(out[i]) for i, k in enumerate(keys)}

    def close(self):
        if self.h:
            self.lib.tioga_b200_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
