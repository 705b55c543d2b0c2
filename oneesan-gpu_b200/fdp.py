"""ctypes binding of libfdp.so, the C ABI in include/oneesan_fdp.h.

This is the Python face of the engine used by the tests and bench.py.  It has
no compute of its own: every call goes through libfdp.so, and loading fails
loudly if the library has not been built (``make -C oneesan-gpu_b200``).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from typing import Sequence

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfdp.so")

FDP_OK = 0
FDP_ERR_ARGS = 1
FDP_ERR_GPU_COUNT = 2
FDP_ERR_WINDOW = 4
FDP_ERR_HBM = 5
FDP_ERR_CUDA = 6
FDP_ERR_MODULUS = 34
FDP_PENDING = 100
FDP_TIMEOUT = 101
FDP_ERR_NOT_FOUND = 102
MAX_LANES = 16
MAX_N = 27


class FdpError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        super().__init__(f"{where}: fdp status {status} {detail}".strip())


class Problem(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("k", ctypes.c_int),
                ("moduli", ctypes.POINTER(ctypes.c_uint32)), ("lanes", ctypes.c_int)]


class PlanOut(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("width", ctypes.c_int), ("k", ctypes.c_int),
                ("lanes", ctypes.c_int), ("passes", ctypes.c_int), ("index_bits", ctypes.c_int),
                ("main_states", ctypes.c_uint64), ("blocked_states", ctypes.c_uint64),
                ("state_bytes", ctypes.c_uint64), ("scratch_bytes", ctypes.c_uint64),
                ("table_bytes", ctypes.c_uint64), ("total_bytes", ctypes.c_uint64),
                ("rows", ctypes.c_int), ("bounded_rows", ctypes.c_int), ("init_rows", ctypes.c_int),
                ("cells_per_row", ctypes.c_int),
                ("alg_bytes_per_residue", ctypes.c_uint64),
                ("transitions_per_residue", ctypes.c_uint64), ("fits", ctypes.c_int),
                ("sweep_peak_bytes", ctypes.c_uint64), ("init_peak_bytes", ctypes.c_uint64)]


class Tuning(ctypes.Structure):
    _fields_ = [("block", ctypes.c_int), ("grid", ctypes.c_int), ("split_panels", ctypes.c_int),
                ("bounded_prefix", ctypes.c_int), ("lane_items", ctypes.c_int), ("share_min", ctypes.c_int),
                ("compact_max_p", ctypes.c_int), ("compact_items", ctypes.c_int),
                ("row_init_rows", ctypes.c_int), ("row_init_product", ctypes.c_int),
                ("split_spans_min_p", ctypes.c_int), ("compact_carry", ctypes.c_int)]


class AutotuneResult(ctypes.Structure):
    _fields_ = [("lanes", ctypes.c_int), ("passes", ctypes.c_int), ("tuning", Tuning),
                ("row_ms", ctypes.c_double), ("s_per_residue", ctypes.c_double),
                ("residues_per_hour", ctypes.c_double), ("candidates", ctypes.c_int),
                ("rejected_memory", ctypes.c_int), ("check_n", ctypes.c_int)]


class RunStats(ctypes.Structure):
    _fields_ = [("wall_s", ctypes.c_double), ("device_s", ctypes.c_double),
                ("capture_s", ctypes.c_double), ("kernel_launches", ctypes.c_uint64),
                ("alg_bytes", ctypes.c_uint64), ("transitions", ctypes.c_uint64)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_uint64), ("max_active", ctypes.c_int),
                ("max_lanes", ctypes.c_int), ("max_bypass_s", ctypes.c_double)]


class RequestInfo(ctypes.Structure):
    _fields_ = [("queue_s", ctypes.c_double), ("run_s", ctypes.c_double), ("latency_s", ctypes.c_double),
                ("device_s", ctypes.c_double), ("lanes", ctypes.c_int), ("passes", ctypes.c_int),
                ("state_bytes", ctypes.c_uint64)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("failed", ctypes.c_uint64),
                ("queued", ctypes.c_uint64), ("running", ctypes.c_uint64), ("pool_bytes", ctypes.c_uint64),
                ("bytes_in_use", ctypes.c_uint64), ("peak_bytes_in_use", ctypes.c_uint64),
                ("peak_running", ctypes.c_int)]


_lib = None


def lib() -> ctypes.CDLL:
    """Load libfdp.so once; raise if it is missing (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libfdp.so not built at {LIB_PATH}; run `make -C oneesan-gpu_b200`")
    L = ctypes.CDLL(LIB_PATH)
    c_int, c_u32, c_u64, c_vp = ctypes.c_int, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_void_p
    P = ctypes.POINTER
    L.fdp_version.restype = ctypes.c_char_p
    L.fdp_last_error.restype = ctypes.c_char_p
    L.fdp_plan.argtypes = [P(Problem), c_u64, P(PlanOut)]
    L.fdp_create.argtypes = [P(c_vp), c_int]
    L.fdp_destroy.argtypes = [c_vp]
    L.fdp_destroy.restype = None
    L.fdp_run_sync.argtypes = [c_vp, P(Problem), P(c_u32), P(RunStats)]
    L.fdp_apply_cells.argtypes = [c_vp, c_int, c_int, c_int, c_int, P(c_u32), c_vp, c_vp, c_vp]
    L.fdp_time_cells.argtypes = [c_vp, P(Problem), c_int, P(ctypes.c_double)]
    L.fdp_set_tuning.argtypes = [c_vp, P(Tuning)]
    L.fdp_get_tuning.argtypes = [c_vp, P(Tuning)]
    L.fdp_autotune.argtypes = [c_vp, P(Problem), c_u64, c_int, P(AutotuneResult), ctypes.c_char_p,
                               ctypes.c_size_t]
    L.fdp_transfer_map_build.argtypes = [c_vp, c_int, c_int, c_int, P(c_vp)]
    L.fdp_transfer_map_info.argtypes = [c_vp, P(c_u64), P(c_u64), P(c_u64)]
    L.fdp_transfer_map_apply.argtypes = [c_vp, c_vp, c_int, P(c_u32), c_vp, c_vp, c_vp, c_vp, c_vp]
    L.fdp_transfer_map_destroy.argtypes = [c_vp]
    L.fdp_transfer_map_destroy.restype = None
    L.fdp_factor_map_build.argtypes = [c_vp, c_int, c_int, c_int, c_int, c_int, c_int, P(c_vp)]
    L.fdp_factor_map_info.argtypes = [c_vp, P(c_u64), P(c_u64), P(c_u64), P(c_u64)]
    L.fdp_factor_map_apply.argtypes = [c_vp, c_vp, c_u32, c_int, P(c_u32), c_vp, c_vp, c_vp, c_vp, c_vp,
                                       P(ctypes.c_double)]
    L.fdp_factor_map_destroy.argtypes = [c_vp]
    L.fdp_factor_map_destroy.restype = None
    L.fdp_reverse2_apply.argtypes = [c_vp, c_int, c_int, c_int, P(c_u32), c_vp, c_vp, c_vp, c_vp, c_vp]
    L.fdp_run_multi_sync.argtypes = [c_vp, P(Problem), c_int, P(c_u32), P(RunStats)]
    L.fdp_server_start.argtypes = [c_vp, P(ServerConfig)]
    L.fdp_server_stop.argtypes = [c_vp]
    L.fdp_submit.argtypes = [c_vp, P(Problem), P(c_u64)]
    L.fdp_poll.argtypes = [c_vp, c_u64, P(c_u32), P(RequestInfo)]
    L.fdp_wait.argtypes = [c_vp, c_u64, c_int, P(c_u32), P(RequestInfo)]
    L.fdp_server_get_stats.argtypes = [c_vp, P(ServerStats)]
    L.fdp_rank_words.argtypes = [c_vp, c_int, c_vp, c_vp, c_u64, c_vp]
    L.fdp_unrank_words.argtypes = [c_vp, c_int, c_vp, c_vp, c_u64, c_vp]
    L.fdp_ternary_index.argtypes = [c_vp, c_vp, c_vp, c_u64, c_vp]
    L.fdp_ternary_index_chunked.argtypes = [c_vp, c_int, c_vp, c_vp, c_u64, c_vp]
    for name in ("fdp_main_states", "fdp_blocked_states"):
        getattr(L, name).argtypes = [c_int]
        getattr(L, name).restype = c_u64
    L.fdp_cell_bytes.argtypes = [c_int, c_int]
    L.fdp_cell_bytes.restype = c_u64
    L.fdp_test_inject_pass_errors.argtypes = [c_int]
    _lib = L
    return L


def _check(status: int, where: str) -> None:
    if status != FDP_OK:
        detail = lib().fdp_last_error().decode(errors="replace")
        raise FdpError(status, where, detail)


def _u32_array(values: Sequence[int]):
    return (ctypes.c_uint32 * len(values))(*[int(v) for v in values])


def lane_panels(lanes: int) -> list:
    """Panels (first lane, width) of the lane layout: greedy widths 8, 4, 2, 1."""
    out, l0 = [], 0
    while l0 < lanes:
        pw = 8 if lanes - l0 >= 8 else 4 if lanes - l0 >= 4 else (2 if lanes - l0 >= 2 else 1)
        out.append((l0, pw))
        l0 += pw
    return out


def lane_spans(lanes: int) -> list:
    """Spans (first lane, end lane) of consecutive panels holding at most 8
    lanes together; a cell of several spans may run as one launch per span."""
    out, l0 = [], 0
    panels = lane_panels(lanes)
    i = 0
    while i < len(panels):
        start, width = panels[i][0], 0
        while i < len(panels) and width + panels[i][1] <= 8:
            width += panels[i][1]
            i += 1
        out.append((start, start + width))
    return out


def pack_lanes(a):
    """(N, lanes) uint32 array -> flat array in the engine's panel layout."""
    import numpy as np
    a = np.ascontiguousarray(a, dtype=np.uint32)
    n, lanes = a.shape
    out = np.empty(n * lanes, dtype=np.uint32)
    for l0, pw in lane_panels(lanes):
        out[l0 * n:(l0 + pw) * n] = a[:, l0:l0 + pw].reshape(-1)
    return out


def unpack_lanes(flat, n: int, lanes: int):
    """Inverse of pack_lanes."""
    import numpy as np
    flat = np.asarray(flat, dtype=np.uint32).reshape(-1)
    out = np.empty((n, lanes), dtype=np.uint32)
    for l0, pw in lane_panels(lanes):
        out[:, l0:l0 + pw] = flat[l0 * n:(l0 + pw) * n].reshape(n, pw)
    return out


def main_states(width: int) -> int:
    return int(lib().fdp_main_states(width))


def blocked_states(width: int) -> int:
    return int(lib().fdp_blocked_states(width))


def cell_bytes(width: int, p: int) -> int:
    return int(lib().fdp_cell_bytes(width, p))


def inject_pass_errors(count: int) -> None:
    """Test hook: the next `count` computations start with their device error
    word set, as when a kernel gives up on a bounded wait."""
    _check(lib().fdp_test_inject_pass_errors(count), "fdp_test_inject_pass_errors")


def plan(n: int, moduli: Sequence[int], lanes: int | None = None, budget: int = 1 << 62) -> PlanOut:
    mods = _u32_array(moduli)
    pr = Problem(n, len(moduli), mods, lanes or min(len(moduli), MAX_LANES))
    out = PlanOut()
    _check(lib().fdp_plan(ctypes.byref(pr), budget, ctypes.byref(out)), "fdp_plan")
    return out


@dataclass
class Result:
    residues: list
    stats: RunStats


class Engine:
    """One engine context on one CUDA device."""

    def __init__(self, device: int = 0):
        self._ctx = ctypes.c_void_p()
        _check(lib().fdp_create(ctypes.byref(self._ctx), device), "fdp_create")

    def close(self) -> None:
        if self._ctx:
            lib().fdp_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def residues(self, n: int, moduli: Sequence[int], lanes: int | None = None) -> Result:
        """Residues of the corner-path count of the n x n grid, one per modulus."""
        mods = _u32_array(moduli)
        pr = Problem(n, len(moduli), mods, lanes or min(len(moduli), MAX_LANES))
        out = (ctypes.c_uint32 * len(moduli))()
        st = RunStats()
        _check(lib().fdp_run_sync(self._ctx, ctypes.byref(pr), out, ctypes.byref(st)), "fdp_run_sync")
        return Result([int(x) for x in out], st)

    def autotune(self, n: int, moduli: Sequence[int], max_lanes: int = MAX_LANES,
                 hbm_budget_bytes: int = 170 * 10**9, repeats: int = 2) -> dict:
        """Pick residues-per-pass, panel strategy and CTA size for (n, moduli);
        the winner is applied to this engine."""
        import json as _json
        mods = _u32_array(moduli)
        pr = Problem(n, len(moduli), mods, max_lanes)
        res = AutotuneResult()
        buf = ctypes.create_string_buffer(1 << 16)
        _check(lib().fdp_autotune(self._ctx, ctypes.byref(pr), hbm_budget_bytes, repeats, ctypes.byref(res), buf,
                                  len(buf)), "fdp_autotune")
        return _json.loads(buf.value.decode())

    def residues_multi(self, problems, lanes: int | None = None):
        """Several (n, moduli) problems in one captured CUDA graph; returns
        ([residues of each problem], RunStats)."""
        keep = [_u32_array(m) for _, m in problems]
        arr = (Problem * len(problems))(*[Problem(n, len(m), keep[i], lanes or min(len(m), MAX_LANES))
                                          for i, (n, m) in enumerate(problems)])
        total = sum(len(m) for _, m in problems)
        out = (ctypes.c_uint32 * total)()
        st = RunStats()
        _check(lib().fdp_run_multi_sync(self._ctx, arr, len(problems), out, ctypes.byref(st)), "fdp_run_multi_sync")
        res, off = [], 0
        for _, m in problems:
            res.append([int(x) for x in out[off:off + len(m)]])
            off += len(m)
        return res, st

    def time_cells(self, n: int, moduli: Sequence[int], lanes: int | None = None, rows: int = 1) -> list:
        """Mean CUDA-event duration (ms) of each cell p = 1..n of a row sweep; index 0 unused."""
        mods = _u32_array(moduli)
        pr = Problem(n, len(moduli), mods, lanes or min(len(moduli), MAX_LANES))
        out = (ctypes.c_double * (n + 1))()
        _check(lib().fdp_time_cells(self._ctx, ctypes.byref(pr), rows, out), "fdp_time_cells")
        return [float(x) for x in out]

    def set_tuning(self, block: int = 256, grid: int = 0, split_panels: bool = False,
                   bounded_prefix: bool = True, lane_items: int = 0, share_min: int = 0,
                   compact_max_p: int = 0, compact_items: int = 0, row_init_rows: int = 0,
                   row_init_product: int = 0, split_spans_min_p: int = 0, compact_carry: int = 0) -> None:
        t = Tuning(block, grid, 1 if split_panels else 0, 1 if bounded_prefix else 0, lane_items, share_min,
                   compact_max_p, compact_items, row_init_rows, row_init_product, split_spans_min_p,
                   compact_carry)
        _check(lib().fdp_set_tuning(self._ctx, ctypes.byref(t)), "fdp_set_tuning")

    def get_tuning(self) -> dict:
        t = Tuning()
        _check(lib().fdp_get_tuning(self._ctx, ctypes.byref(t)), "fdp_get_tuning")
        return {"block": t.block, "grid": t.grid, "split_panels": bool(t.split_panels),
                "bounded_prefix": bool(t.bounded_prefix), "lane_items": t.lane_items, "share_min": t.share_min,
                "compact_max_p": t.compact_max_p, "compact_items": t.compact_items,
                "row_init_rows": t.row_init_rows, "row_init_product": t.row_init_product,
                "split_spans_min_p": t.split_spans_min_p, "compact_carry": t.compact_carry}

    # ---- serving -------------------------------------------------------------
    def server_start(self, hbm_budget_bytes: int, max_active: int = 8, max_lanes: int = 16,
                     max_bypass_s: float = 30.0) -> None:
        cfg = ServerConfig(hbm_budget_bytes, max_active, max_lanes, max_bypass_s)
        _check(lib().fdp_server_start(self._ctx, ctypes.byref(cfg)), "fdp_server_start")

    def server_stop(self) -> None:
        _check(lib().fdp_server_stop(self._ctx), "fdp_server_stop")

    def submit(self, n: int, moduli: Sequence[int]) -> int:
        mods = _u32_array(moduli)
        pr = Problem(n, len(moduli), mods, 1)
        rid = ctypes.c_uint64()
        _check(lib().fdp_submit(self._ctx, ctypes.byref(pr), ctypes.byref(rid)), "fdp_submit")
        self._pending_k = getattr(self, "_pending_k", {})
        self._pending_k[rid.value] = len(moduli)
        return rid.value

    def _result(self, rid: int, status: int, out, info):
        if status == FDP_PENDING or status == FDP_TIMEOUT:
            return None
        self._pending_k.pop(rid, None)
        _check(status, "request")
        return {"residues": [int(x) for x in out], "queue_s": info.queue_s, "run_s": info.run_s,
                "latency_s": info.latency_s, "device_s": info.device_s, "lanes": info.lanes,
                "passes": info.passes, "state_bytes": info.state_bytes}

    def poll(self, rid: int):
        """Result dict, or None while the request is queued or running."""
        out = (ctypes.c_uint32 * self._pending_k[rid])()
        info = RequestInfo()
        return self._result(rid, lib().fdp_poll(self._ctx, rid, out, ctypes.byref(info)), out, info)

    def wait(self, rid: int, timeout_ms: int = 600000):
        """Result dict, or None if the bounded wait ran out."""
        out = (ctypes.c_uint32 * self._pending_k[rid])()
        info = RequestInfo()
        return self._result(rid, lib().fdp_wait(self._ctx, rid, timeout_ms, out, ctypes.byref(info)), out, info)

    def server_stats(self) -> dict:
        st = ServerStats()
        _check(lib().fdp_server_get_stats(self._ctx, ctypes.byref(st)), "fdp_server_get_stats")
        return {f: getattr(st, f) for f, _ in ServerStats._fields_}

    # ---- operator variants ---------------------------------------------------
    def transfer_map(self, width: int, p: int, paired: bool = False) -> "TransferMap":
        h = ctypes.c_void_p()
        _check(lib().fdp_transfer_map_build(self._ctx, width, p, 1 if paired else 0, ctypes.byref(h)),
               "fdp_transfer_map_build")
        return TransferMap(self, h)

    def factor_map(self, width: int, p: int, fixed: int, occupied: int, paired: bool = False,
                   max_groups: int = 32) -> "FactorMap":
        h = ctypes.c_void_p()
        _check(lib().fdp_factor_map_build(self._ctx, width, p, 1 if paired else 0, fixed, occupied, max_groups,
                                          ctypes.byref(h)), "fdp_factor_map_build")
        return FactorMap(self, h)

    def reverse2_apply(self, width: int, p: int, moduli: Sequence[int], in_main: int, in_block: int,
                       out_main: int, out_block: int, stream: int = 0) -> None:
        mods = _u32_array(moduli)
        _check(lib().fdp_reverse2_apply(self._ctx, width, p, len(moduli), mods, in_main, in_block, out_main,
                                        out_block, stream), "fdp_reverse2_apply")

    def apply_cells(self, width: int, p_hi: int, p_lo: int, moduli: Sequence[int], main_ptr: int,
                    block_ptr: int, stream: int = 0) -> None:
        mods = _u32_array(moduli)
        _check(lib().fdp_apply_cells(self._ctx, width, p_hi, p_lo, len(moduli), mods, main_ptr, block_ptr,
                                     stream), "fdp_apply_cells")

    def rank_words(self, width: int, words_ptr: int, ranks_ptr: int, count: int, stream: int = 0) -> None:
        _check(lib().fdp_rank_words(self._ctx, width, words_ptr, ranks_ptr, count, stream), "fdp_rank_words")

    def unrank_words(self, width: int, ranks_ptr: int, words_ptr: int, count: int, stream: int = 0) -> None:
        _check(lib().fdp_unrank_words(self._ctx, width, ranks_ptr, words_ptr, count, stream), "fdp_unrank_words")

    def ternary_index(self, codes_ptr: int, index_ptr: int, count: int, stream: int = 0) -> None:
        _check(lib().fdp_ternary_index(self._ctx, codes_ptr, index_ptr, count, stream), "fdp_ternary_index")

    def ternary_index_chunked(self, chunk: int, codes_ptr: int, index_ptr: int, count: int, stream: int = 0) -> None:
        _check(lib().fdp_ternary_index_chunked(self._ctx, chunk, codes_ptr, index_ptr, count, stream),
               "fdp_ternary_index_chunked")


class TransferMap:
    """A CSR transfer map on the device (fdp_transfer_map_*)."""

    def __init__(self, engine: Engine, handle):
        self._eng, self._h = engine, handle

    def info(self) -> dict:
        r, e, b = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        _check(lib().fdp_transfer_map_info(self._h, ctypes.byref(r), ctypes.byref(e), ctypes.byref(b)),
               "fdp_transfer_map_info")
        return {"rows": r.value, "edges": e.value, "device_bytes": b.value}

    def apply(self, moduli: Sequence[int], in_main: int, in_block: int, out_main: int, out_block: int,
              stream: int = 0) -> None:
        mods = _u32_array(moduli)
        _check(lib().fdp_transfer_map_apply(self._eng._ctx, self._h, len(moduli), mods, in_main, in_block,
                                            out_main, out_block, stream), "fdp_transfer_map_apply")

    def close(self) -> None:
        if self._h:
            lib().fdp_transfer_map_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class FactorMap:
    """A CSR over one occupancy-group shape, applied to many conjugate groups
    (fdp_factor_map_*)."""

    def __init__(self, engine: Engine, handle):
        self._eng, self._h = engine, handle

    def info(self) -> dict:
        gm, gd, e, b = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        _check(lib().fdp_factor_map_info(self._h, ctypes.byref(gm), ctypes.byref(gd), ctypes.byref(e),
                                         ctypes.byref(b)), "fdp_factor_map_info")
        return {"group_main": gm.value, "group_blocked": gd.value, "edges": e.value, "device_bytes": b.value}

    def apply(self, modulus: int, masks: Sequence[int], in_main: int, in_block: int, out_main: int,
              out_block: int, stream: int = 0, timed: bool = False):
        """Apply to the groups `masks`; returns [gather, apply, scatter] ms when timed."""
        m = _u32_array(masks)
        ph = (ctypes.c_double * 3)() if timed else None
        _check(lib().fdp_factor_map_apply(self._eng._ctx, self._h, modulus, len(masks), m, in_main, in_block,
                                          out_main, out_block, stream, ph), "fdp_factor_map_apply")
        return [float(x) for x in ph] if timed else None

    def close(self) -> None:
        if self._h:
            lib().fdp_factor_map_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
