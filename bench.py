#!/usr/bin/env python
"""Benchmark of the TIOGA overset-connectivity path on B200.

One step = one tioga_performconnectivity_ call (hole maps, box pairs, query
gathering, donor search with Newton containment, donor selection and
cancellation, final iblanks) on the mixed-element workload: a 257^3 Cartesian
background whose z<0 hexes are split into prisms, plus three 65x65x129
spherical shells whose first four radial layers are split into tets, prisms
and pyramids (seeded synthetic mesh, 18.5 M nodes, 27 M cells).

The metric unit is the query point (a receptor-candidate node handed to a
donor search), as in the reference's own bookkeeping (the nsearch lists).

  value   device-resident inputs (coordinates already in HBM), split-precision
          search, aggregate over all GPUs (replicas: each GPU runs its own
          system, no data-path collective)
  plain   the same with FP64 arithmetic throughout (the plain GPU form)
  e2e     through the C ABI with the caller's host buffers: coordinates copied
          host->device and iblank device->host inside every step
  latency_ms  p50/p99 of the per-step device time (split form)

  python bench.py [--gpus N --steps K --warmup W]
  python bench.py --impl reference      # the compiled reference on the CPU
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from tioga_b200 import cases  # noqa: E402
from tioga_b200.capi import TiogaLibrary  # noqa: E402

METRIC = "connectivity receptors/s & p99 latency vs plain GPU form, 0 iblank/donor mismatch"
UNIT = "receptors/s"
WORKLOAD0 = ("cfg0: 65^3 all-hex background on [-5,5]^3 + one all-hex spherical shell 33x33x65 (radii 0.5-2.0, "
             "radial stretching 1.1), interior nodes perturbed by 5% of the spacing")
WORKLOAD = ("cfg1: 257^3 background (z<0 hexes split into 2 prisms) + 3 spherical shells "
            "65x65x129 (first 4 radial layers split into tets/prisms/pyramids), seed 1")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libtioga_ref.so")
PORT_LIB = os.path.join(ROOT, "oracle", "_ref", "liboracle.so")
# DRAM bytes (read + write) of one k_cell_boxes launch per cell, from an ncu
# capture on the full workload (profiles/k_cell_boxes_cfg1.md).
CELL_BOX_DRAM_BYTES_PER_CELL = 2235169536 / 26961129  # 82.90 B


def cell_box_bytes(system, st):
    """Compulsory bytes of one k_cell_boxes launch (the split form's cell and
    leaf boxes), each array read or written once: per cell its vertex
    references (4 B each, the reference's connectivity), its type (1 B) read
    and its FP32 box (24 B) written; per node its FP32 copy (16 B, made by
    k_node_tiles outside this launch) read once; per leaf its record (16 B)
    read and its box (24 B) written."""
    nvsum = sum(nv * conn.shape[0] for b in system.blocks for nv, conn in b.cells)
    return 4 * nvsum + 16 * system.nnodes + system.ncells * (1 + 24) + st["nleaf"] * (16 + 24)


# bounded CPU sample: the same geometry at 97^3 background and 25x25x49 shells
CPU_SAMPLE = dict(nbg=97, nshell=3, nr=25, nt=25, nphi=49, split_layers=4)
CPU_SAMPLE_TEXT = ("cfg1 geometry at reduced resolution (97^3 background, three 25x25x49 shells, "
                   "4 split layers): one connectivity call per sample")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=50)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="tioga_b200", choices=["tioga_b200", "reference"])
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--ref-systems", type=int, default=16,
                   help="--impl reference with cfg2/cfg3: systems of the distribution in the CPU sample")
    p.add_argument("--no-cpu-full", action="store_true",
                   help="skip the one full-size connectivity call of the compiled reference")
    p.add_argument("--no-parity", action="store_true",
                   help="skip the mismatch count against the compiled reference's digests")
    p.add_argument("--cpu-reps", type=int, default=3)
    p.add_argument("--size", default="full", choices=["full", "medium", "small"],
                   help="cfg1 at full size, at 161^3 + 49x49x97 shells (profiling), or at test size")
    p.add_argument("--workload", default="cfg1", choices=["cfg0", "cfg1", "cfg2", "cfg3", "cfg4"],
                   help="cfg0: the small all-hex system, CPU-runnable at full size (its reference arm times it "
                        "whole); cfg1: one mixed-element system (default); cfg2: the batched form, 64 systems; "
                        "cfg3: the serving form, Poisson requests over resident moving systems; "
                        "cfg4: the high-order path, degree-3 Lagrange shell over a degree-1 background")
    p.add_argument("--rates", default="",
                   help="cfg3: comma-separated arrival rates (requests/s); default: a sweep around capacity")
    p.add_argument("--seconds", type=float, default=6.0, help="cfg3: arrival window per rate")
    p.add_argument("--slots", type=int, default=8, help="cfg3: concurrent requests")
    p.add_argument("--nsys", type=int, default=200, help="cfg3: systems")
    p.add_argument("--budget-gb", type=float, default=120.0, help="cfg3: HBM admission budget")
    p.add_argument("--fields", default="host", choices=["host", "device"],
                   help="cfg3: the requests' 5 fields in pinned host memory or on the device")
    p.add_argument("--no-tune", action="store_true", help="keep the default launch shapes (no autotuning)")
    p.add_argument("--tuning", default="",
                   help="launch shapes by hand instead of the autotuner, tioga_b200_tuning_'s order: cell-pass "
                        "CTAs/SM, pairs per cell-pass CTA, query CTAs/SM, traversal CTAs/SM, candidate CTAs/SM, "
                        "cell-box CTAs/SM, traversal variant + 1 (1: leaves as met, 2: leaves postponed); e.g. 3,128,16,64,16,6,2")
    p.add_argument("--no-forms", action="store_true",
                   help="cfg1: skip the batched (cfg2) and served (cfg3) summaries added to the line")
    p.add_argument("--forms", default="split,plain,e2e,e2e_pageable",
                   help="comma list of measured forms (the first one gives `value`)")
    return p.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing (one process per GPU, replicas)
# ---------------------------------------------------------------------------
def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Dist:
    def __init__(self, ws, device):
        self.ws = ws
        self.pg = None
        if ws > 1:
            import datetime

            import torch.distributed as dist
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=device)
            self.pg = dist

    def barrier(self):
        if self.pg:
            import torch
            self.pg.barrier(device_ids=[torch.cuda.current_device()])

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v: float) -> float:
        if not self.pg:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: str):
        self.index = index
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.index, f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for n, v in zip(names, f[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def pinned_copy(system):
    """The caller's arrays in pinned host memory (coordinates and iblank)."""
    import torch
    blocks, ibls, keep = [], [], []
    for b in system.blocks:
        xt = torch.empty((b.nnodes, 3), dtype=torch.float64, pin_memory=True)
        xt.numpy()[:] = b.x
        it = torch.ones(b.nnodes, dtype=torch.int32, pin_memory=True)
        keep += [xt, it]
        blocks.append(cases.Block(b.tag, xt.numpy(), b.cells, b.wbc, b.obc, b.name))
        ibls.append(it.numpy())
    return cases.System(blocks, system.name, system.meta), ibls, keep


def set_tuning(lib, text: str):
    v = [int(t) for t in text.split(",")]
    v += [0] * (7 - len(v))
    lib.lib.tioga_b200_set_tuning_((C.c_int * 7)(*v[:7]))


def autotune(lib, tb, reps: int = 2) -> dict:
    """The library's autotuner (tioga_b200_autotune_) on the loaded workload;
    returns the launch shapes it chose."""
    tb.set_int(lib.lib, "tioga_b200_autotune_", reps)
    if lib.lib.tioga_b200_last_error() != 0:
        raise RuntimeError("autotune failed")
    return read_tuning(lib)


def read_tuning(lib) -> dict:
    """The launch shapes in use (tioga_b200_tuning_)."""
    out = (C.c_int * 8)()
    lib.lib.tioga_b200_tuning_(out)
    keys = ["cell_pass_ctas_per_sm", "pairs_per_cell_pass_cta", "query_ctas_per_sm", "traverse_ctas_per_sm",
            "candidate_ctas_per_sm", "cell_box_ctas_per_sm", "traverse_variant"]
    return {k: int(out[i]) for i, k in enumerate(keys)}


GOLDEN = os.path.join(ROOT, "tests", "golden")


def parity_vs_reference(lib, tb, system, fixture: str, q_seed: int, precisions=(1, 0)):
    """Mismatches of the timed configuration against the compiled reference's
    digests (tests/golden/make_digests.py): iblank per node, getdonorinfo
    records per record, updated fields per 4096 values, for each precision
    form, after one more connectivity call with the caller's host iblank
    arrays.  None when no fixture covers this configuration."""
    from tests.golden import digest
    path = os.path.join(GOLDEN, fixture + ".npz")
    if not os.path.exists(path):
        return None
    fix = np.load(path)
    if digest.input_digest(system) != str(fix["input_digest"]):
        return {"error": "the generated mesh differs from the fixture's"}
    q0 = cases.fields(system, nvar=5, seed=q_seed)
    out = {"against": f"compiled reference, digests in tests/golden/{fixture}.npz", "forms": {}}
    for b in system.blocks:
        lib.lib.tioga_b200_registeriblank_device_(C.byref(C.c_int(b.tag)), C.c_void_p(0))
    total = 0
    for prec in precisions:
        tb.set_int(lib.lib, "tioga_b200_set_precision_", prec)
        lib.performconnectivity()
        res = {"iblank": {}, "donors": {}, "q": {}}
        for b in system.blocks:
            res["iblank"][b.tag] = lib.iblank(b.tag).copy()
            res["donors"][b.tag] = lib.getdonorinfo(b.tag)
        qs = [np.array(q, dtype=np.float64, copy=True) for q in q0]
        for b, q in zip(system.blocks, qs):
            lib.registersolution(b.tag, q)
        lib.dataupdate_mb(5, "row")
        for b, q in zip(system.blocks, qs):
            res["q"][b.tag] = q
        c = digest.compare(fix, system, res)
        st = tb.stats(lib.lib)
        name = {0: "fp64", 1: "split"}.get(prec, str(prec))
        out["forms"][name] = {"iblank_mismatches": c["iblank"], "record_mismatches": c["records"],
                              "records": c["record_total"], "field_chunk_mismatches": c["q_chunks"],
                              "ties": st["nties"]}
        total += c["iblank"] + c["records"] + c["q_chunks"]
    out["mismatches"] = total
    out["ties"] = max(f["ties"] for f in out["forms"].values())
    return out


def run_gpu(args, ws, rank, local, dist):
    import torch

    import tioga_b200 as tb
    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    if args.workload == "cfg0":
        system = cases.small_config0(args.seed) if args.size == "small" else cases.config0(args.seed)
    elif args.size == "small":
        system = cases.small_config1(args.seed)
    elif args.size == "medium":
        system = cases.config1(args.seed, nbg=161, nshell=3, nr=49, nt=49, nphi=97, split_layers=4)
    else:
        system = cases.config1(args.seed)
    psys, ibls, keep = pinned_copy(system)
    lib = TiogaLibrary(tb.library_path())
    tb.extras(lib.lib)
    lib.init()
    if lib.lib.tioga_b200_last_error() != 0:
        raise RuntimeError("libtioga_b200 could not initialise the GPU")
    lib.register_system(psys, ibls)
    lib.lib.tioga_b200_set_stream_(C.c_void_p(stream.cuda_stream))
    tb.set_int(lib.lib, "tioga_b200_set_precision_", 1)
    lib.preprocess_grids()
    lib.performconnectivity()
    if lib.lib.tioga_b200_last_error() != 0:
        raise RuntimeError("connectivity failed")
    if args.tuning:
        set_tuning(lib, args.tuning)
    tuning = read_tuning(lib) if (args.no_tune or args.tuning) else autotune(lib, tb)

    # device-resident forms keep iblank in HBM too (a GPU solver's arrays)
    d_ibl = [torch.ones(b.nnodes, dtype=torch.int32, device="cuda") for b in system.blocks]

    def timed(precision, resident, steps, warmup, clocks=None):
        tb.set_int(lib.lib, "tioga_b200_set_precision_", precision)
        tb.set_int(lib.lib, "tioga_b200_set_coords_resident_", resident)
        for b, d in zip(system.blocks, d_ibl):
            lib.lib.tioga_b200_registeriblank_device_(C.byref(C.c_int(b.tag)),
                                                       C.c_void_p(d.data_ptr() if resident else 0))
        for _ in range(warmup):
            lib.performconnectivity()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        phases, launches = [], 0
        dist.barrier()
        torch.cuda.synchronize()
        if clocks:
            clocks.start()
        ev[0].record(stream)
        for k in range(steps):
            lib.performconnectivity()
            ev[k + 1].record(stream)
            phases.append(tb.timing(lib.lib))
            launches += tb.stats(lib.lib)["launches"]
        torch.cuda.synchronize()
        clk = clocks.stop() if clocks else None
        dist.barrier()
        if lib.lib.tioga_b200_last_error() != 0:
            raise RuntimeError("connectivity failed during timing")
        per = [ev[k].elapsed_time(ev[k + 1]) for k in range(steps)]
        total = dist.max(ev[0].elapsed_time(ev[steps]))
        st = tb.stats(lib.lib)
        avg = {k: float(np.mean([p[k] for p in phases])) for k in phases[0]}
        return total / steps, per, st, avg, launches, clk

    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    idx = vis.split(",")[local] if vis else str(local)
    clocks = Clocks(idx)
    forms = args.forms.split(",")
    ms_split, per_split, st, ph, launches, clk = timed(1, 1, args.steps, args.warmup, clocks)
    Q = st["nquery"]
    if "plain" in forms:
        ms_plain, per_plain, st_plain, ph_plain, _, _ = timed(0, 1, args.steps, args.warmup)
        assert st_plain["nquery"] == Q
    else:
        ms_plain, per_plain = float("nan"), [float("nan")]
    if "e2e" in forms:
        ms_e2e, per_e2e, st_e2e, ph_e2e, _, _ = timed(1, 0, args.steps, args.warmup)
        assert st_e2e["nquery"] == Q
    else:
        ms_e2e = float("nan")
    h2d = sum(24 * b.nnodes for b in system.blocks)
    d2h = sum(4 * b.nnodes for b in system.blocks)
    # Roofline kernel: k_cell_boxes, the cell pass's pass over every cell (one
    # launch per step; cell_box_bytes gives its compulsory bytes).
    cell_ms = ph["cell_boxes"]
    nvsum = sum(nv * conn.shape[0] for b in system.blocks for nv, conn in b.cells)
    alg_bytes = cell_box_bytes(system, st)
    traffic = (None if CELL_BOX_DRAM_BYTES_PER_CELL is None
               else CELL_BOX_DRAM_BYTES_PER_CELL * system.ncells)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = alg_bytes / (cell_ms * 1e-3) / 1e9
    out = {
        "metric": METRIC, "value": ws * Q / (ms_split * 1e-3), "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_split, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded mesh generator tioga_b200.cases)",
        "config": {"workload": (WORKLOAD0 if args.workload == "cfg0" else WORKLOAD) if args.size == "full"
                   else f"{args.workload} geometry, {args.size} size",
                   "nodes": system.nnodes, "cells": system.ncells, "blocks": len(system.blocks),
                   "query_points": Q, "receptors": st["nreceptor"], "holes": st["nhole"],
                   "precision": "fp32 Newton screen + fp64 refinement",
                   "parallelism": f"replicas x{ws}",
                   "l2": "inputs larger than L2 (coordinates %.0f MB, connectivity %.0f MB)" % (
                       h2d / 1e6, sum(32 * b.ncells for b in system.blocks) / 1e6)},
        "latency_ms": {"p50": float(np.percentile(per_split, 50)), "p99": float(np.percentile(per_split, 99)),
                       "max": float(np.max(per_split))},
        "plain": {"value": ws * Q / (ms_plain * 1e-3), "ms_per_step": ms_plain,
                  "p99_ms": float(np.percentile(per_plain, 99)), "precision": "fp64 throughout"},
        "speedup_vs_plain": ms_plain / ms_split,
        "e2e": {"value": ws * Q / (ms_e2e * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": ms_e2e},
        "roofline": {"kernel": "k_cell_boxes (FP32 cell and leaf boxes)", "bound": "hbm",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "algorithmic_bytes": alg_bytes, "launch_ms": cell_ms,
                     "pairs_kernel_ms": ph["cell_pass"] - ph["cell_boxes"],
                     "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"},
        "phases_ms": ph,
        "search": {"candidates": st["ncand"], "fp64_refinements": st["nrefine"], "ties": st["nties"],
                   "donors": st["ndonor"]},
        "tuning": tuning,
        "gpu_launches": launches,
        "clocks": clk,
    }
    # parity of the timed configuration against the compiled reference
    if args.workload == "cfg1" and args.size == "full" and args.seed == 1 and not args.no_parity:
        out["parity"] = parity_vs_reference(lib, tb, psys, "cfg1_full", 21)
    # the whole call against its compulsory bytes (B_conn): every array of the
    # path read or written once -- coordinates, connectivity, cell and node
    # resolutions, iblanks, cell iblanks, hole maps, query buffers and their
    # sort keys, donor ids and interpolation records
    tb.set_int(lib.lib, "tioga_b200_set_precision_", 1)
    tb.set_int(lib.lib, "tioga_b200_set_coords_resident_", 1)
    lib.performconnectivity()
    st2 = (C.c_longlong * 8)()
    lib.lib.tioga_b200_stats2_(st2)
    nw1 = sum(int((lib.getdonorinfo(b.tag)[0][:, 3] + 1).sum()) for b in system.blocks)
    N, Cc, R = system.nnodes, system.ncells, st["nreceptor"]
    b_conn = (24 * N + 4 * nvsum + 8 * Cc + 8 * N + 4 * N + 4 * Cc + int(st2[0]) + Q * (24 + 8) + Q * (24 + 4)
              + 4 * R + 12 * nw1)
    out["roofline"]["call"] = {"algorithmic_bytes": b_conn, "ms": ms_split,
                               "achieved": b_conn / (ms_split * 1e-3) / 1e9,
                               "frac": b_conn / (ms_split * 1e-3) / 1e9 / peak,
                               "note": "the whole connectivity call (split form, resident coordinates) against "
                                       "its compulsory bytes"}
    out["dataupdate"] = time_dataupdate(lib, system, stream, st["nreceptor"], args.steps, args.warmup)
    lib.lib.tioga_b200_set_stream_(C.c_void_p(0))
    lib.delete()
    del keep
    if "e2e_pageable" in forms:
        out["e2e_pageable"] = time_e2e_pageable(system, stream, args.steps, args.warmup, ws)
    out["_system"] = system
    return out


def time_e2e_pageable(system, stream, steps: int, warmup: int, ws: int):
    """e2e with the caller's arrays in ordinary pageable memory (numpy), as a
    Fortran or C solver would pass them: the library page-locks them at its
    first preprocess (tioga_b200_set_pin_host_, on by default), so every
    later call copies at the pinned rate."""
    import torch

    import tioga_b200 as tb
    lib = TiogaLibrary(tb.library_path())
    tb.extras(lib.lib)
    lib.init()
    lib.register_system(system)  # numpy arrays: pageable host memory
    lib.lib.tioga_b200_set_stream_(C.c_void_p(stream.cuda_stream))
    tb.set_int(lib.lib, "tioga_b200_set_precision_", 1)
    t0 = time.perf_counter()
    lib.preprocess_grids()
    pin_s = time.perf_counter() - t0
    for _ in range(max(1, warmup)):
        lib.performconnectivity()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        lib.performconnectivity()
    e1.record(stream)
    torch.cuda.synchronize()
    err = lib.lib.tioga_b200_last_error()
    Q = tb.stats(lib.lib)["nquery"]
    lib.lib.tioga_b200_set_stream_(C.c_void_p(0))
    lib.delete()
    if err:
        return {"error": f"connectivity failed ({err})"}
    ms = e0.elapsed_time(e1) / steps
    return {"value": ws * Q / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
            "first_preprocess_s": pin_s,
            "note": "caller arrays in pageable memory, page-locked by the library at its first preprocess"}


def time_dataupdate(lib, system, stream, nreceptor: int, steps: int, warmup: int, nvar: int = 5):
    """The data update after the last connectivity call, reported on its own
    as receptor-fields per second: 5 FP64 fields per node in the ROW layout,
    resident on the device (a GPU solver's arrays), CUDA events around
    `steps` calls after `warmup` untimed ones."""
    import torch
    try:
        dq = [torch.empty(b.nnodes * nvar, dtype=torch.float64, device="cuda").uniform_(-1.0, 1.0)
              for b in system.blocks]
        for b, d in zip(system.blocks, dq):
            lib.lib.tioga_b200_registersolution_device_(C.byref(C.c_int(b.tag)), C.c_void_p(d.data_ptr()))
        for _ in range(max(1, warmup)):
            lib.dataupdate_mb(nvar, "row")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            lib.dataupdate_mb(nvar, "row")
        e1.record(stream)
        torch.cuda.synchronize()
        if lib.lib.tioga_b200_last_error() != 0:
            return {"error": "data update failed"}
        ms = e0.elapsed_time(e1) / steps
        return {"ms": ms, "receptors": nreceptor, "nvar": nvar, "layout": "row, fields on the device",
                "receptor_fields_per_s": nreceptor * nvar / (ms * 1e-3)}
    except Exception as ex:  # the connectivity line stands without it
        return {"error": repr(ex)}


# ---------------------------------------------------------------------------
# batched form: 64 independent systems in one instance
# ---------------------------------------------------------------------------
WORKLOAD2 = ("cfg2: 64 independent overset systems (background box + 1-4 spherical shells, node counts "
             "log-uniform in [5e4, 2e6], all-hex or mixed-element with p=0.5), seed 2, one instance")


def batch_systems(args, rank: int = 0, ws: int = 1):
    """The batch's systems, and on N GPUs this rank's share of them: systems
    are independent, so they are dealt round-robin to the ranks with no
    exchange between GPUs (strong scaling of the batch)."""
    if args.size == "small":
        allsys = cases.config2(2, nsys=8, nmin=5e3, nmax=5e4)
    elif args.size == "medium":
        allsys = cases.config2(2, nsys=16, nmin=2e4, nmax=5e5)
    else:
        allsys = cases.config2(2)
    return shard(allsys, rank, ws)


def shard(items, rank: int, ws: int):
    """Round-robin share of rank `rank` among `ws` ranks."""
    return list(items[rank::ws])


def run_gpu_batch(args, ws, rank, local, dist):
    """The batched form against the plain form on the same systems: every
    system in one instance (one launch per stage over all of them) versus one
    system per instance, one after another (the reference's way of running
    independent systems)."""
    import torch

    import tioga_b200 as tb
    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    systems = batch_systems(args, rank, ws)
    pinned = [pinned_copy(s) for s in systems]
    lib = TiogaLibrary(tb.library_path())
    tb.extras(lib.lib)
    lib.lib.tioga_b200_nsystems_.restype = C.c_int

    def events_time(steps, warmup, clocks=None):
        for _ in range(warmup):
            lib.performconnectivity()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        phases, launches = [], 0
        dist.barrier()
        torch.cuda.synchronize()
        if clocks:
            clocks.start()
        ev[0].record(stream)
        for k in range(steps):
            lib.performconnectivity()
            ev[k + 1].record(stream)
            phases.append(tb.timing(lib.lib))
            launches += tb.stats(lib.lib)["launches"]
        torch.cuda.synchronize()
        clk = clocks.stop() if clocks else None
        dist.barrier()
        if lib.lib.tioga_b200_last_error() != 0:
            raise RuntimeError("connectivity failed during timing")
        per = [ev[k].elapsed_time(ev[k + 1]) for k in range(steps)]
        avg = {k: float(np.mean([p[k] for p in phases])) for k in phases[0]}
        return ev[0].elapsed_time(ev[steps]) / steps, per, tb.stats(lib.lib), avg, launches, clk

    # plain form: one system per instance, one after another
    forms = args.forms.split(",")
    plain_ms = {0: float("nan"), 1: float("nan")}
    plain_q = None
    for (psys, ibls, _keep) in (pinned if "plain" in forms else []):
        if plain_q is None:
            plain_ms, plain_q = {0: 0.0, 1: 0.0}, 0
        lib.init()
        lib.register_system(psys, ibls)
        lib.lib.tioga_b200_set_stream_(C.c_void_p(stream.cuda_stream))
        tb.set_int(lib.lib, "tioga_b200_set_coords_resident_", 1)
        lib.preprocess_grids()
        for prec in (1, 0):
            tb.set_int(lib.lib, "tioga_b200_set_precision_", prec)
            ms, _, st, _, _, _ = events_time(max(1, args.steps // 2), 1)
            plain_ms[prec] += ms
        plain_q += st["nquery"]
        lib.lib.tioga_b200_set_stream_(C.c_void_p(0))
        lib.delete()
    # batched form
    lib.init()
    for k, (psys, ibls, _keep) in enumerate(pinned):
        for bid, (b, ib) in enumerate(zip(psys.blocks, ibls), start=1):
            lib.select_system(k)
            lib.registergrid_data_mb(bid, b, ib)
    assert lib.lib.tioga_b200_nsystems_() == len(systems)
    lib.lib.tioga_b200_set_stream_(C.c_void_p(stream.cuda_stream))
    tb.set_int(lib.lib, "tioga_b200_set_precision_", 1)
    lib.preprocess_grids()
    d_ibl = []
    for k, s in enumerate(systems):
        lib.select_system(k)
        for b in s.blocks:
            d = torch.ones(b.nnodes, dtype=torch.int32, device="cuda")
            d_ibl.append(d)
            lib.lib.tioga_b200_registeriblank_device_(C.byref(C.c_int(b.tag)), C.c_void_p(d.data_ptr()))
    tb.set_int(lib.lib, "tioga_b200_set_coords_resident_", 1)
    if args.tuning:
        set_tuning(lib, args.tuning)
    tuning = read_tuning(lib) if (args.no_tune or args.tuning) else autotune(lib, tb)
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    clocks = Clocks(vis.split(",")[local] if vis else str(local))
    ms_b, per_b, st, ph, launches, clk = events_time(args.steps, args.warmup, clocks)
    Q = st["nquery"]
    assert plain_q is None or Q == plain_q, (Q, plain_q)
    ms_b64 = ms_e2e = float("nan")
    if "plain" in forms:
        tb.set_int(lib.lib, "tioga_b200_set_precision_", 0)
        ms_b64, _, st64, _, _, _ = events_time(max(1, args.steps // 2), 1)
        assert st64["nquery"] == Q
    # end to end: host coordinates in, host iblanks out, every step
    if "e2e" in forms:
        tb.set_int(lib.lib, "tioga_b200_set_precision_", 1)
        tb.set_int(lib.lib, "tioga_b200_set_coords_resident_", 0)
        for k, s in enumerate(systems):
            lib.select_system(k)
            for b in s.blocks:
                lib.lib.tioga_b200_registeriblank_device_(C.byref(C.c_int(b.tag)), C.c_void_p(0))
        ms_e2e, _, st_e, _, _, _ = events_time(args.steps, args.warmup)
        assert st_e["nquery"] == Q
    nodes = sum(s.nnodes for s in systems)
    cells = sum(s.ncells for s in systems)
    h2d, d2h = 24 * nodes, 4 * nodes
    cell_ms = ph["cell_boxes"]
    nvsum = sum(nv * conn.shape[0] for s in systems for b in s.blocks for nv, conn in b.cells)
    alg_bytes = cell_box_bytes(cases.System([b for sy in systems for b in sy.blocks]), st)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = alg_bytes / (cell_ms * 1e-3) / 1e9
    # on N GPUs every rank connects its share of the systems: the job's rate
    # is all ranks' query points over the slowest rank's time
    q_all = dist.sum(float(Q))
    ms_job = dist.max(ms_b)
    out = {
        "metric": METRIC, "value": q_all / (ms_job * 1e-3), "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_job, "higher_is_better": True,
        "scaling": "strong" if ws > 1 else "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded mesh generator tioga_b200.cases.config2)",
        "config": {"workload": WORKLOAD2 if args.size == "full" else f"cfg2 distribution, {args.size} size",
                   "systems": len(systems), "nodes": nodes, "cells": cells,
                   "blocks": sum(len(s.blocks) for s in systems), "query_points": Q,
                   "receptors": st["nreceptor"], "holes": st["nhole"],
                   "precision": "fp32 Newton screen + fp64 refinement",
                   "parallelism": f"systems dealt round-robin to {ws} GPUs, no exchange" if ws > 1 else "1 GPU",
                   "l2": "inputs larger than L2 (coordinates %.0f MB)" % (h2d / 1e6)},
        "latency_ms": {"p50": float(np.percentile(per_b, 50)), "p99": float(np.percentile(per_b, 99)),
                       "max": float(np.max(per_b))},
        "plain": {"value": ws * Q / (plain_ms[0] * 1e-3), "ms_per_step": plain_ms[0],
                  "form": "one system per instance, one after another, fp64 throughout"},
        "plain_split": {"value": ws * Q / (plain_ms[1] * 1e-3), "ms_per_step": plain_ms[1],
                        "form": "one system per instance, one after another, split precision"},
        "batched_fp64": {"value": ws * Q / (ms_b64 * 1e-3), "ms_per_step": ms_b64},
        "speedup_vs_plain": plain_ms[0] / ms_b,
        "e2e": {"value": ws * Q / (ms_e2e * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": ms_e2e},
        "roofline": {"kernel": "k_cell_boxes (FP32 cell and leaf boxes)", "bound": "hbm",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": (None if CELL_BOX_DRAM_BYTES_PER_CELL is None
                                 else CELL_BOX_DRAM_BYTES_PER_CELL * cells), "algorithmic_bytes": alg_bytes,
                     "launch_ms": cell_ms, "pairs_kernel_ms": ph["cell_pass"] - ph["cell_boxes"],
                     "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"},
        "phases_ms": ph,
        "search": {"candidates": st["ncand"], "fp64_refinements": st["nrefine"], "ties": st["nties"],
                   "donors": st["ndonor"]},
        "tuning": tuning,
        "gpu_launches": launches,
        "clocks": clk,
    }
    lib.lib.tioga_b200_set_stream_(C.c_void_p(0))
    lib.delete()
    return out


# ---------------------------------------------------------------------------
# serving form: Poisson requests over resident moving systems
# ---------------------------------------------------------------------------
WORKLOAD3 = ("cfg3: Poisson request stream over {n} resident systems from the cfg2 distribution (seed 3); each "
             "request one time step of one system: every shell rotated U(0,2) degrees about a random axis and "
             "moved by <= 0.5 wall-layer cell widths, then preprocess, connectivity and a 5-field data update")


def serving_systems(args):
    n = args.nsys
    if args.size == "small":
        return cases.config2(3, nsys=min(n, 16), nmin=5e3, nmax=5e4)
    if args.size == "medium":
        return cases.config2(3, nsys=min(n, 48), nmin=2e4, nmax=5e5)
    return cases.config2(3, nsys=n)


def wall_cell_width(block) -> float:
    """The smallest edge of the cells that touch the block's wall."""
    wall = np.zeros(block.nnodes, dtype=bool)
    wall[block.wbc] = True
    best = np.inf
    for nv, conn in block.cells:
        c = conn[wall[conn].any(axis=1)]
        if len(c) == 0:
            continue
        p = block.x[c]
        e = np.linalg.norm(p[:, 1:, :] - p[:, :1, :], axis=2)
        e = e[e > 0]
        if e.size:
            best = min(best, float(e.min()))
    return best if np.isfinite(best) else 0.0


def run_gpu_serving(args, ws, rank, local, dist):
    import torch

    from tioga_b200.serving import Server, rigid
    torch.cuda.set_device(local)
    systems = serving_systems(args)
    nvar = 5
    rng = np.random.default_rng(33)
    pinned, keep = [], []
    for s in systems:  # the solver's arrays in pinned host memory
        xs, ibs, qs = [], [], []
        for b in s.blocks:
            xt = torch.empty((b.nnodes, 3), dtype=torch.float64, pin_memory=True)
            xt.numpy()[:] = b.x
            it = torch.ones(b.nnodes, dtype=torch.int32, pin_memory=True)
            qt = torch.empty(b.nnodes * nvar, dtype=torch.float64, pin_memory=True)
            qt.numpy()[:] = rng.uniform(-1.0, 1.0, b.nnodes * nvar)
            if args.fields == "device":
                qt = qt.cuda()
            keep += [xt, it, qt]
            xs.append(xt.numpy())
            ibs.append(it.numpy())
            qs.append(qt if args.fields == "device" else qt.numpy())
        pinned.append((xs, ibs, qs))
    shift = [[0.5 * wall_cell_width(b) for b in s.blocks] for s in systems]
    srv = Server(budget_bytes=int(args.budget_gb * (1 << 30)), nslots=args.slots, max_resident=200)
    for k, s in enumerate(systems):
        srv.add_system(k, s, x_arrays=pinned[k][0], ibl_arrays=pinned[k][1])

    def fields(k):
        key = "q_device" if args.fields == "device" else "q"
        return {key: pinned[k][2], "nvar": nvar}

    def moves_for(k):
        s = systems[k]
        xs = pinned[k][0]
        return [(b.tag, *rigid(rng, xs[i][:: max(1, b.nnodes // 64)].mean(axis=0), 2.0, shift[k][i]))
                for i, b in enumerate(s.blocks) if i > 0]

    # admission: one step of every system (topology upload, trees, hole maps)
    t0 = time.perf_counter()
    ts = [srv.submit(k, moves_for(k), **fields(k)) for k in range(len(systems))]
    first = [srv.wait(t) for t in ts]
    admit_s = time.perf_counter() - t0
    assert all(f["rc"] == 0 for f in first), [f for f in first if f["rc"]][:3]
    # a closed loop with all slots busy measures the capacity
    t0 = time.perf_counter()
    ts = [srv.submit(k % len(systems), moves_for(k % len(systems)), **fields(k % len(systems)))
          for k in range(2 * len(systems))]
    sat = [srv.wait(t) for t in ts]
    sat_s = time.perf_counter() - t0
    cap = len(ts) / sat_s
    rates = [float(r) for r in args.rates.split(",")] if args.rates else [0.25 * cap, 0.5 * cap, 0.75 * cap,
                                                                          0.9 * cap]
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    clocks = Clocks(vis.split(",")[local] if vis else str(local))
    sweep = []
    for ri, rate in enumerate(rates):
        n = max(8, int(rate * args.seconds))
        arr = np.cumsum(rng.exponential(1.0 / rate, n))
        who = rng.integers(0, len(systems), n)
        mv = [moves_for(int(k)) for k in who]
        if ri == len(rates) - 1:
            clocks.start()
        tickets = []
        t0 = time.perf_counter()
        for i in range(n):  # submit at the arrival times
            d = t0 + arr[i] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            tickets.append(srv.submit(int(who[i]), mv[i], **fields(int(who[i]))))
        res = [srv.wait(t) for t in tickets]
        wall = time.perf_counter() - t0
        clk = clocks.stop() if ri == len(rates) - 1 else None
        assert all(r["rc"] == 0 for r in res)
        lat = np.array([r["latency_ms"] for r in res])
        Q = sum(r["nquery"] for r in res)
        sweep.append({"rate_rps": rate, "requests": n, "seconds": wall, "receptors_per_s": Q / wall,
                      "requests_per_s": n / wall, "query_points": Q,
                      "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                                     "p99.9": float(np.percentile(lat, 99.9)), "max": float(lat.max())},
                      "queue_ms_p50": float(np.median([r["queue_ms"] for r in res])),
                      "service_ms_p50": float(np.median([r["service_ms"] for r in res])),
                      "calls_ms_p50": {k: float(np.median([r[k + "_ms"] for r in res]))
                                       for k in ("preprocess", "connectivity", "dataupdate")}})
    st = srv.stats()
    srv.close()
    top = sweep[-1]
    nodes = sum(s.nnodes for s in systems)
    # on N GPUs every rank serves its own stream of requests: the rates add up
    job_rate = dist.sum(top["receptors_per_s"])
    out = {
        "metric": METRIC, "value": job_rate, "unit": UNIT, "n_gpus": ws, "steps": top["requests"],
        "warmup": len(systems), "ms_per_step": 1e3 * top["seconds"] / top["requests"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded mesh generator tioga_b200.cases.config2, seeded rigid motions)",
        "config": {"workload": WORKLOAD3.format(n=len(systems)) if args.size == "full" else
                   f"cfg3 stream, {args.size} systems", "systems": len(systems), "nodes": nodes,
                   "slots": args.slots, "budget_gb": args.budget_gb, "arrivals": "Poisson",
                   "fields": args.fields,
                   "parallelism": f"replicas x{ws}",
                   "l2": "inputs larger than L2 (all systems' coordinates %.0f MB)" % (24 * nodes / 1e6)},
        "latency_ms": top["latency_ms"],
        "serving": {"capacity_rps": cap, "capacity_receptors_per_s": sum(r["nquery"] for r in sat) / sat_s,
                    "admission_s": admit_s, "sweep": sweep, "server": st},
        "e2e": {"value": top["receptors_per_s"], "unit": UNIT,
                "h2d_bytes_per_step": 0 if args.fields == "device" else int(np.mean([8 * nvar * s.nnodes
                                                                                      for s in systems])),
                "d2h_bytes_per_step": int(np.mean([(4 + (0 if args.fields == "device" else 8 * nvar)) * s.nnodes
                                                   for s in systems])),
                "note": "requests through the serving C ABI; every request downloads its system's iblanks "
                        "and, with host fields, uploads its fields and downloads the interpolated values"},
        "gpu_launches": None,
        "clocks": clk,
    }
    del keep
    return out


# ---------------------------------------------------------------------------
# high-order path: degree-3 Lagrange shell over a degree-1 background
# ---------------------------------------------------------------------------
WORKLOAD4 = ("cfg4: 97^3 degree-1 background + a curved spherical-shell band of 24x24x48 degree-3 Lagrange "
             "hexahedra (64 DOFs each), interior DOFs perturbed +-2%, seed 4; one step = performconnectivity + "
             "performconnectivity_highorder; a seeded cubic field (5 variables) for the data update")


def run_gpu_highorder(args, ws, rank, local, dist):
    import torch

    import tioga_b200 as tb
    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    if args.size == "small":
        system, ho = cases.config4(4, nbg=33, ne_r=6, ne_t=8, ne_p=16)
    elif args.size == "medium":
        system, ho = cases.config4(4, nbg=65, ne_r=12, ne_t=12, ne_p=24)
    else:
        system, ho = cases.config4(4)
    nvar = 5
    lib = TiogaLibrary(tb.library_path())
    tb.extras(lib.lib)
    lib.init()
    lib.register_system(system)
    xd = [np.ascontiguousarray(h.xdof, dtype=np.float64) for h in ho]
    for b, h, x in zip(system.blocks, ho, xd):
        lib.lib.tioga_b200_set_highorder_lagrange_(C.byref(C.c_int(b.tag)), C.byref(C.c_int(h.p)),
                                                   x.ctypes.data_as(C.c_void_p))
    lib.lib.tioga_b200_set_stream_(C.c_void_p(stream.cuda_stream))
    tb.set_int(lib.lib, "tioga_b200_set_coords_resident_", 1)
    lib.preprocess_grids()

    def hostats():
        st = (C.c_longlong * 8)()
        lib.lib.tioga_b200_highorder_stats_(st)
        return list(st)

    def timed(prec, steps, warmup, resident=1):
        tb.set_int(lib.lib, "tioga_b200_set_precision_", prec)
        tb.set_int(lib.lib, "tioga_b200_set_coords_resident_", resident)
        for _ in range(warmup):
            lib.performconnectivity()
            lib.lib.tioga_performconnectivity_highorder_()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        torch.cuda.synchronize()
        ev[0].record(stream)
        for k in range(steps):
            lib.performconnectivity()
            lib.lib.tioga_performconnectivity_highorder_()
            ev[k + 1].record(stream)
        torch.cuda.synchronize()
        if lib.lib.tioga_b200_last_error() != 0:
            raise RuntimeError("high-order connectivity failed")
        per = [ev[k].elapsed_time(ev[k + 1]) for k in range(steps)]
        return ev[0].elapsed_time(ev[steps]) / steps, per, hostats()

    def update():
        q0 = cases.dof_fields(ho, nvar, seed=5)  # the cubic at every DOF
        q = [a.copy() for a in q0]
        for b, a in zip(system.blocks, q):
            lib.registersolution(b.tag, a)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        lib.dataupdate_mb(nvar, "row")
        e1.record(stream)
        torch.cuda.synchronize()
        return q0, q, e0.elapsed_time(e1)

    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    clocks = Clocks(vis.split(",")[local] if vis else str(local))
    clocks.start()
    ms_split, per_split, st_split = timed(1, args.steps, args.warmup)
    clk = clocks.stop()
    q0, q_split, upd_ms = update()
    forms = args.forms.split(",")
    if "plain" in forms:
        ms_fp64, per_fp64, st_fp64 = timed(0, max(2, args.steps // 2), 1)
        _, q_fp64, _ = update()
        ms_scr, _, st_scr = timed(2, max(2, args.steps // 2), 1)
        _, q_scr, _ = update()
        scr_vs_fp64 = max(float(np.max(np.abs(a - b))) if a.size else 0.0 for a, b in zip(q_scr, q_fp64))
    else:
        ms_fp64, st_fp64, q_fp64, ms_scr, st_scr, scr_vs_fp64 = float("nan"), st_split, q_split, float("nan"), \
            st_split, float("nan")
    ms_e2e = timed(1, max(2, args.steps // 2), 1, resident=0)[0] if "e2e" in forms else float("nan")
    h2d = 24 * system.nnodes + sum(24 * h.xdof.shape[0] * h.xdof.shape[1] for h in ho)
    Q = st_split[0]
    assert st_fp64[0] == Q
    changed = np.concatenate([(a != b) for a, b in zip(q_split, q0)])
    split_vs_fp64 = max(float(np.max(np.abs(a - b))) if a.size else 0.0 for a, b in zip(q_split, q_fp64))
    interp_err = max(float(np.max(np.abs(a - b))) if a.size else 0.0 for a, b in zip(q_split, q0))
    ms_job = dist.max(ms_split)  # replicas: every rank runs the whole workload
    out = {
        "metric": METRIC, "value": ws * Q / (ms_job * 1e-3), "unit": UNIT + " (high-order query points)",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_split,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded mesh generator tioga_b200.cases.config4, seeded cubic field)",
        "config": {"workload": WORKLOAD4 if args.size == "full" else f"cfg4 geometry, {args.size} size",
                   "nodes": system.nnodes, "cells": system.ncells,
                   "shell_elements": int(ho[1].xdof.shape[0]), "dofs_per_element": int(ho[1].xdof.shape[1]),
                   "highorder_query_points": Q, "parallelism": f"replicas x{ws}"},
        "latency_ms": {"p50": float(np.percentile(per_split, 50)), "p99": float(np.percentile(per_split, 99))},
        "plain": {"value": ws * Q / (ms_fp64 * 1e-3), "ms_per_step": ms_fp64, "precision": "fp64 throughout"},
        "speedup_vs_plain": ms_fp64 / ms_split,
        "e2e": {"value": ws * Q / (ms_e2e * 1e-3), "unit": UNIT, "ms_per_step": ms_e2e, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": 4 * system.nnodes,
                "note": "corner and DOF coordinates uploaded from the caller's arrays every step"},
        "inclusion_tests": {"split": {"tests": st_split[6], "fp64_decided": st_split[7]},
                            "fp64": {"tests": st_fp64[6], "fp64_decided": st_fp64[7]},
                            "fp32_screen": {"tests": st_scr[6], "fp64_decided": st_scr[7], "ms_per_step": ms_scr,
                                            "max_abs_vs_fp64": scr_vs_fp64}},
        "point_donors": st_split[1], "ties": st_split[2], "records": st_split[3],
        "dataupdate": {"ms": upd_ms, "updated_values": int(changed.sum())},
        "errors": {"split_vs_fp64_max_abs": split_vs_fp64,
                   "note": "the FP64 form is bit-identical to the oracle (tests/test_gpu_highorder.py), so "
                           "split_vs_fp64 is the error against the FP64 oracle",
                   "cubic_field_max_abs": interp_err,
                   "cubic_note": "updated DOF values against the cubic they sample: the interpolation error of "
                                 "the donors (curved isoparametric and trilinear elements do not reproduce a "
                                 "cubic in x, y, z exactly)"},
        "gpu_launches": None,
        "clocks": clk,
    }
    lib.lib.tioga_b200_set_stream_(C.c_void_p(0))
    lib.delete()
    return out


# ---------------------------------------------------------------------------
# CPU: the compiled reference (or the C restatement) on a bounded sample
# ---------------------------------------------------------------------------
def sample_query_count(sample):
    """Q of the sample, from the C restatement's query lists (identical to the
    reference's; cheap next to the timed calls)."""
    t = TiogaLibrary(PORT_LIB)
    t.init()
    t.register_system(sample)
    t.preprocess_grids()
    t.performconnectivity()
    ns, nd, tot = C.c_int(), C.c_int(), 0
    for b in sample.blocks:
        t.lib.tioga_oracle_searchstats(C.c_int(b.tag), C.byref(ns), C.byref(nd))
        tot += ns.value
    t.delete()
    return tot


def cpu_reference(reps: int, warmup: int = 1, whole_cfg0: bool = False):
    lib = REF_LIB if os.path.exists(REF_LIB) else PORT_LIB
    kind = "reference" if lib == REF_LIB else "port"
    if not os.path.exists(lib):
        return None, "no CPU build of the reference or the port (run `make -C oracle`)"
    sample = cases.config0(1) if whole_cfg0 else cases.config1(1, **CPU_SAMPLE)
    Q = sample_query_count(sample)
    t = TiogaLibrary(lib)
    t.init()
    t.register_system(sample)
    t.preprocess_grids()
    for _ in range(warmup):
        t.performconnectivity()
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        t.performconnectivity()
        times.append(time.perf_counter() - t0)
    t.delete()
    mean = float(np.mean(times))
    return {"value": Q / mean, "unit": UNIT, "cores": 1, "kind": kind,
            "sample": ("the whole cfg0 system, seed 1" if whole_cfg0 else CPU_SAMPLE_TEXT)
            + f" (Q={Q} query points, {reps} timed calls, mean {mean:.2f} s)",
            "per_step_s": times}, None


def cpu_reference_full(system):
    """One full-size connectivity call of the compiled reference on the timed
    configuration itself (after its preprocess), on one host core: the rate per
    query point at full size, beside the bounded sample's."""
    if not os.path.exists(REF_LIB):
        return None
    sys.path.insert(0, ROOT)
    from tests.golden import digest
    t = TiogaLibrary(REF_LIB)
    t.init()
    t.register_system(system)
    t0 = time.perf_counter()
    t.preprocess_grids()
    t1 = time.perf_counter()
    t.performconnectivity()
    t2 = time.perf_counter()
    t.delete()
    Q = None
    fix = os.path.join(GOLDEN, "cfg1_full.npz")
    if os.path.exists(fix):
        f = np.load(fix)
        if digest.input_digest(system) == str(f["input_digest"]):
            Q = int(f["query_points"][0])
    return {"preprocess_s": t1 - t0, "connectivity_s": t2 - t1, "query_points": Q,
            "value": (Q / (t2 - t1)) if Q else None, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": "the full timed configuration, one connectivity call"}


def _ref_batch_worker(job):
    """One process of the batched/served CPU baseline: the compiled reference
    runs its share of the systems one after another (the reference's way of
    running independent systems, one instance at a time)."""
    kind, nsys, seed, share, steps, nvar = job
    sys.path.insert(0, ROOT)
    from tioga_b200.serving import apply_rigid, rigid
    systems = cases.config2(seed, nsys=nsys)
    rng = np.random.default_rng(1000 + share[0] if share else 0)
    out = []
    for k in share:
        s = systems[k]
        t = TiogaLibrary(REF_LIB)
        t.init()
        t.register_system(s)
        if kind == "cfg2":
            t0 = time.perf_counter()
            t.preprocess_grids()
            t1 = time.perf_counter()
            t.performconnectivity()
            t2 = time.perf_counter()
            out.append({"system": k, "preprocess_s": t1 - t0, "connectivity_s": t2 - t1})
        else:  # one request = a time step: rigid motions, preprocess, connectivity, data update
            qs = [rng.uniform(-1.0, 1.0, b.nnodes * nvar) for b in s.blocks]
            for _ in range(steps):
                t0 = time.perf_counter()
                for i, b in enumerate(s.blocks[1:], start=1):
                    x = t.blocks[b.tag]["x"].reshape(-1, 3)
                    A, bb = rigid(rng, x[:: max(1, b.nnodes // 64)].mean(axis=0), 2.0, 0.0)
                    x[:] = apply_rigid(x, A, bb)
                t.preprocess_grids()
                t.performconnectivity()
                for b, q in zip(s.blocks, qs):  # after the connectivity call, as the reference wants
                    t.registersolution(b.tag, q)
                t.dataupdate_mb(nvar, "row")
                out.append({"system": k, "request_s": time.perf_counter() - t0})
        t.delete()
    return out


def cpu_reference_batch(kind: str, nsys: int = 16, steps: int = 2, procs: int = 0):
    """The batched (cfg2) or served (cfg3) workload on the CPU: the compiled
    reference on a sample of `nsys` systems of the distribution, the systems
    dealt round-robin to P independent processes (P = the host's cores, at
    most nsys), rates summed: query points over the slowest process's busy
    time.  Query counts come from the digest fixture of the first 16 cfg2
    systems (cfg2) or from the oracle's query lists (cfg3)."""
    import multiprocessing as mp
    if not os.path.exists(REF_LIB):
        return None, "the compiled reference is not built (make -C oracle ref)"
    P = max(1, min(procs or os.cpu_count() or 1, nsys))
    seed = 2 if kind == "cfg2" else 3
    jobs = [(kind, nsys, seed, list(range(r, nsys, P)), steps, 5) for r in range(P)]
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(P) as pool:
        parts = pool.map(_ref_batch_worker, jobs)
    wall = time.perf_counter() - t0
    if kind == "cfg2":
        fix = np.load(os.path.join(GOLDEN, "cfg2_16.npz"))
        qp = [int(v) for v in fix["query_points"]]
        if nsys > len(qp):
            return None, "query counts are stored for the first 16 systems only"
        busy = [sum(r["connectivity_s"] for r in part) for part in parts]
        Q = sum(qp[:nsys])
        return {"value": Q / max(busy), "unit": UNIT, "cores": P, "kind": "reference",
                "sample": f"the first {nsys} systems of the cfg2 distribution, one connectivity call each, "
                          f"dealt to {P} processes (rates summed: all query points over the busiest process's "
                          f"connectivity time)",
                "query_points": Q, "busiest_process_s": max(busy), "wall_s": wall,
                "preprocess_s": sum(r["preprocess_s"] for part in parts for r in part)}, None
    systems = cases.config2(seed, nsys=nsys)
    qsys = []
    for s in systems:  # Q per request (rigid motions change it little; the unmoved count stands in)
        t = TiogaLibrary(PORT_LIB)
        t.init()
        t.register_system(s)
        t.preprocess_grids()
        t.performconnectivity()
        ns, nd, tot = C.c_int(), C.c_int(), 0
        for b in s.blocks:
            t.lib.tioga_oracle_searchstats(C.c_int(b.tag), C.byref(ns), C.byref(nd))
            tot += ns.value
        t.delete()
        qsys.append(tot)
    lat = [r["request_s"] for part in parts for r in part]
    busy = [sum(r["request_s"] for r in part) for part in parts]
    Q = sum(qsys[r["system"]] for part in parts for r in part)
    return {"value": Q / max(busy), "unit": UNIT, "cores": P, "kind": "reference",
            "sample": f"{nsys} systems of the cfg3 distribution, {steps} requests each (rigid motion, preprocess, "
                      f"connectivity, 5-field data update), dealt to {P} processes",
            "requests_per_s": len(lat) / max(busy),
            "latency_ms": {"p50": 1e3 * float(np.percentile(lat, 50)), "p99": 1e3 * float(np.percentile(lat, 99))},
            "wall_s": wall}, None


def main():
    args = parse()
    ws, rank, local = dist_env()
    if args.impl == "reference":
        if rank != 0:
            return 0
        if args.workload in ("cfg2", "cfg3"):
            res, why = cpu_reference_batch(args.workload, nsys=args.ref_systems, steps=args.steps)
            if res is None:
                print(json.dumps({"impl": "reference", "unavailable": why}))
                return 0
            print(json.dumps({"impl": "reference", "metric": METRIC, "value": res["value"], "unit": UNIT,
                              "n_gpus": ws, "higher_is_better": True, "dtype": "f64",
                              "config": {"workload": WORKLOAD2 if args.workload == "cfg2" else
                                         WORKLOAD3.format(n=args.ref_systems), "sample": res["sample"]},
                              "cpu_baseline": res,
                              "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}))
            return 0
        res, why = cpu_reference(args.steps, args.warmup, whole_cfg0=(args.workload == "cfg0"))
        if res is None:
            print(json.dumps({"impl": "reference", "unavailable": why}))
            return 0
        line = {"impl": "reference", "metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * float(np.mean(res["per_step_s"])), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded mesh generator tioga_b200.cases)",
                "config": {"workload": WORKLOAD0 if args.workload == "cfg0" else WORKLOAD, "sample": res["sample"]},
                "cpu_baseline": {k: res[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0
    dev = None
    if ws > 1:  # one GPU per rank, set before the process group binds it
        import torch
        torch.cuda.set_device(local)
        dev = torch.device("cuda", local)
    dist = Dist(ws, dev)
    try:
        out = {"cfg2": run_gpu_batch, "cfg3": run_gpu_serving,
               "cfg4": run_gpu_highorder}.get(args.workload, run_gpu)(args, ws, rank, local, dist)
    finally:
        dist.close()
    if rank == 0 and ws == 1 and args.workload == "cfg1" and not args.no_forms:
        # the other two forms on their own workloads, summarised in the same line
        import copy
        a2 = copy.copy(args)
        a2.steps, a2.warmup = max(3, min(args.steps, 6)), max(3, min(args.warmup, 3))
        b = run_gpu_batch(a2, ws, rank, local, Dist(1, None))
        out["batched"] = {k: b[k] for k in ("value", "unit", "ms_per_step", "speedup_vs_plain", "latency_ms",
                                            "plain", "plain_split", "batched_fp64", "e2e", "phases_ms", "roofline",
                                            "tuning", "gpu_launches", "clocks")}
        out["batched"]["config"] = b["config"]
        a3 = copy.copy(args)
        # the cfg3 stream itself (200 resident systems), 2 s per arrival rate
        a3.size, a3.seconds, a3.slots, a3.rates, a3.nsys = "full", 2.0, 16, "", 200
        sv = run_gpu_serving(a3, ws, rank, local, Dist(1, None))
        out["served"] = {k: sv[k] for k in ("value", "unit", "latency_ms", "serving", "e2e", "clocks")}
        out["served"]["config"] = sv["config"]
    system = out.pop("_system", None)
    if rank == 0 and ws == 1 and args.workload == "cfg1" and "batched" in out and "served" in out:
        # the north-star comparison as worded: the split-precision batched and
        # served forms against the plain (FP64, single-system) form at cfg1 scale
        plain = out["plain"]["value"]
        best = max(out["batched"]["value"], out["served"]["serving"]["capacity_receptors_per_s"])
        par = out.get("parity") or {}
        forms = par.get("forms", {})
        out["north_star"] = {
            "plain_fp64_cfg1": plain, "split_cfg1": out["value"], "split_batched_cfg2": out["batched"]["value"],
            "served_capacity": out["served"]["serving"]["capacity_receptors_per_s"],
            "served_p99_ms": out["served"]["latency_ms"]["p99"],
            "ratio_best_vs_plain": best / plain, "target_ratio": 3.0, "met": best / plain >= 3.0,
            "mismatches": par.get("mismatches"), "ties": par.get("ties"),
            "max_weight_error_vs_fp64": (0.0 if forms and all(f["record_mismatches"] == 0 and
                                                             f["field_chunk_mismatches"] == 0
                                                             for f in forms.values()) else None),
            "note": "weights and updated fields of both forms equal the reference's digests bit for bit, so the "
                    "split form's weight error against FP64 is 0"}
    if rank == 0:
        if ws == 1 and not args.no_cpu_baseline:
            res, why = cpu_reference(args.cpu_reps, whole_cfg0=(args.workload == "cfg0"))
            out["cpu_baseline"] = ({k: res[k] for k in ("value", "unit", "cores", "kind", "sample")}
                                   if res else {"unavailable": why})
            if res and system is not None and args.workload == "cfg1" and args.size == "full" \
                    and not args.no_cpu_full:
                out["cpu_baseline"]["full_size"] = cpu_reference_full(system)
        else:
            out["cpu_baseline"] = None
        print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
