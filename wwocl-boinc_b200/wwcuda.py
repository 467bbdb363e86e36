"""ctypes binding of libwwcuda.so (include/wwcuda.h) for Python callers.

This is the Python face of the C ABI that the wwocl host program uses; the
tests and the benchmark drive the CUDA path through it.  There is no CPU
fallback: importing this module fails when the shared library is missing,
and every call raises WWError on a non-zero status.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libwwcuda.so"

if not LIB_PATH.exists():
    raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {PKG}` (no CPU fallback exists)")

_L = C.CDLL(str(LIB_PATH))

WW_OK = 0
STATUS = {0: "ok", -1: "cuda", -2: "arg", -3: "prp_overflow", -4: "hit_overflow", -5: "timeout",
          -6: "nomem", -7: "composite", -8: "state", -9: "nodev"}


class WWError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = _L.ww_last_error().decode(errors="replace")
        super().__init__(f"{where}: {STATUS.get(status, status)} ({msg})")
        self.status = status


class Hit(C.Structure):
    _fields_ = [("p", C.c_uint64), ("result", C.c_int32), ("rem", C.c_int32),
                ("quot", C.c_int32), ("pad", C.c_int32)]


class Counters(C.Structure):
    _fields_ = [("checksum", C.c_uint64), ("total_prp_count", C.c_uint64),
                ("result_count", C.c_uint32), ("seg_prp_count", C.c_uint32),
                ("max_prp_count", C.c_uint32), ("overflow", C.c_uint32)]


class Buffers(C.Structure):
    _fields_ = [("prime", C.c_void_p), ("invert", C.c_void_p), ("one", C.c_void_p),
                ("special_prime", C.c_void_p), ("rem", C.c_void_p), ("quot", C.c_void_p),
                ("result", C.c_void_p), ("checksum", C.c_void_p), ("total_prp_count", C.c_void_p),
                ("result_count", C.c_void_p), ("primecount", C.c_void_p), ("overflow", C.c_void_p),
                ("prp_capacity", C.c_uint64), ("hit_capacity", C.c_uint32), ("stream", C.c_void_p)]


class Unit(C.Structure):
    _fields_ = [("start", C.c_uint64), ("end", C.c_uint64)]


class UnitResult(C.Structure):
    _fields_ = [("checksum", C.c_uint64), ("prp_count", C.c_uint64), ("hits", C.c_uint32),
                ("tiles_done", C.c_uint32)]


class BatchCfg(C.Structure):
    _fields_ = [("seg_words", C.c_uint32), ("threads", C.c_uint32), ("ppt", C.c_uint32),
                ("joint", C.c_uint32)]

    def as_tuple(self):
        return (self.seg_words, self.threads, self.ppt, self.joint)


class Request(C.Structure):
    _fields_ = [("id", C.c_uint64), ("start", C.c_uint64), ("end", C.c_uint64)]


class RequestResult(C.Structure):
    _fields_ = [("id", C.c_uint64), ("checksum", C.c_uint64), ("prp_count", C.c_uint64),
                ("prps_stored", C.c_uint64), ("hits", C.c_uint32), ("status", C.c_int32),
                ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double)]


class ServerCfg(C.Structure):
    _fields_ = [("prp_pool_bytes", C.c_uint64), ("max_active", C.c_uint32), ("epoch_tiles", C.c_uint32),
                ("max_hits", C.c_uint32), ("store_prps", C.c_uint32)]


class State(C.Structure):
    _fields_ = [("current", C.c_uint64), ("cksm", C.c_uint64), ("psum", C.c_double), ("pcnt", C.c_int32),
                ("pad", C.c_int32)]


_U64P = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_VP = C.c_void_p
_SIGS = {
    "ww_last_error": (C.c_char_p, []),
    "ww_status_string": (C.c_char_p, [C.c_int]),
    "ww_abi_version": (C.c_int, []),
    "ww_launch_clearn": (C.c_int, [_VP, _VP]),
    "ww_launch_clearresult": (C.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "ww_launch_getsegprimes": (C.c_int, [C.c_uint64, C.c_uint64, C.c_int32, _VP, _VP, _VP, C.c_uint64,
                                         _VP, _VP]),
    "ww_launch_wieferich": (C.c_int, [_VP] * 11 + [C.c_uint64, C.c_uint32, _VP, _VP]),
    "ww_launch_wallsunsun": (C.c_int, [_VP] * 10 + [C.c_uint64, C.c_uint32, _VP, _VP]),
    "ww_launch_test_prps": (C.c_int, [_VP] * 10 + [C.c_uint64, C.c_uint32, _VP, _VP]),
    "ww_launch_digits": (C.c_int, [_VP, C.c_uint64, _VP, _VP]),
    "ww_open": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "ww_close": (None, [_VP]),
    "ww_reserve": (C.c_int, [_VP, C.c_uint64, C.c_uint32]),
    "ww_clear_results": (C.c_int, [_VP]),
    "ww_clear_segment": (C.c_int, [_VP]),
    "ww_sieve_prp": (C.c_int, [_VP, C.c_uint64, C.c_uint64, C.c_int32]),
    "ww_set_sieve_depth": (C.c_int, [_VP, C.c_int]),
    "ww_get_sieve_depth": (C.c_int, [_VP, C.POINTER(C.c_int)]),
    "ww_selftest_deep_table": (C.c_int, [_VP, C.c_int, C.c_uint64, C.c_uint64, _VP, _VP,
                                         C.POINTER(C.c_uint64)]),
    "ww_set_sieve_shape": (C.c_int, [_VP, C.c_int]),
    "ww_get_sieve_shape": (C.c_int, [_VP, C.POINTER(C.c_int)]),
    "ww_wieferich": (C.c_int, [_VP]),
    "ww_wallsunsun": (C.c_int, [_VP]),
    "ww_test_prps": (C.c_int, [_VP]),
    "ww_load_prps": (C.c_int, [_VP, _VP, C.c_uint64]),
    "ww_test_prps_host": (C.c_int, [_VP, _VP, C.c_uint64]),
    "ww_count_prps": (C.c_int, [_VP, C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64)]),
    "ww_marker": (C.c_int, [_VP, C.c_int]),
    "ww_wait_marker": (C.c_int, [_VP, C.c_int, C.c_uint32]),
    "ww_marker_elapsed": (C.c_int, [_VP, C.c_int, C.c_int, C.POINTER(C.c_float)]),
    "ww_sync": (C.c_int, [_VP, C.c_uint32]),
    "ww_read_counters": (C.c_int, [_VP, C.POINTER(Counters)]),
    "ww_read_hits": (C.c_int, [_VP, C.POINTER(Hit), C.c_uint32, C.POINTER(C.c_uint32)]),
    "ww_read_prps": (C.c_int, [_VP, _VP, C.c_uint64, C.POINTER(C.c_uint64)]),
    "ww_get_buffers": (C.c_int, [_VP, C.POINTER(Buffers)]),
    "ww_find_wheel_offset": (C.c_int, [C.POINTER(C.c_uint64), C.POINTER(C.c_int32)]),
    "ww_is_prime": (C.c_int, [C.c_uint64]),
    "ww_is_prp": (C.c_int, [C.c_uint64]),
    "ww_parse_number": (C.c_int, [C.c_char_p, C.POINTER(C.c_uint64)]),
    "ww_format_hits": (C.c_int, [C.POINTER(Hit), C.c_uint32, C.c_char_p, C.c_size_t,
                                 C.POINTER(C.c_uint32)]),
    "ww_prp_count_bound": (C.c_uint64, [C.c_uint64, C.c_uint64]),
    "ww_state_write": (C.c_int, [C.c_char_p, C.c_char_p, C.c_uint64, C.c_uint64, C.POINTER(State),
                                 C.POINTER(C.c_int)]),
    "ww_state_read": (C.c_int, [C.c_char_p, C.c_char_p, C.c_uint64, C.c_uint64, C.POINTER(State),
                                C.POINTER(C.c_int)]),
    "ww_selftest_digits": (C.c_int, [_U64P, C.c_uint64, _U64P]),
    "ww_selftest_range": (C.c_int, [C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64),
                                    C.POINTER(C.c_uint64), C.POINTER(C.c_uint32)]),
    "ww_batch_configs": (C.c_int, [C.POINTER(BatchCfg), C.c_uint32, C.POINTER(C.c_uint32)]),
    "ww_batch_set_config": (C.c_int, [_VP, C.POINTER(BatchCfg)]),
    "ww_batch_get_config": (C.c_int, [_VP, C.POINTER(BatchCfg)]),
    "ww_batch_reserve_hits": (C.c_int, [_VP, C.c_uint32]),
    "ww_batch_submit": (C.c_int, [_VP, C.POINTER(Unit), C.c_uint32]),
    "ww_batch_collect": (C.c_int, [_VP, C.POINTER(UnitResult), C.c_uint32, C.POINTER(C.c_uint32)]),
    "ww_batch_run": (C.c_int, [_VP, C.POINTER(Unit), C.c_uint32, C.POINTER(UnitResult)]),
    "ww_batch_hits": (C.c_int, [_VP, C.POINTER(Hit), C.POINTER(C.c_uint32), C.c_uint32,
                                C.POINTER(C.c_uint32)]),
    "ww_batch_tune": (C.c_int, [_VP, C.POINTER(Unit), C.c_uint32, C.POINTER(BatchCfg),
                                C.POINTER(C.c_float)]),
    "ww_server_open": (C.c_int, [_VP, C.POINTER(ServerCfg)]),
    "ww_server_close": (C.c_int, [_VP]),
    "ww_server_submit": (C.c_int, [_VP, C.POINTER(Request), C.c_uint32]),
    "ww_server_step": (C.c_int, [_VP, C.POINTER(RequestResult), C.c_uint32, C.POINTER(C.c_uint32)]),
    "ww_server_status": (C.c_int, [_VP, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]),
    "ww_server_hits": (C.c_int, [_VP, C.c_uint64, C.POINTER(Hit), C.c_uint32, C.POINTER(C.c_uint32)]),
    "ww_server_prps": (C.c_int, [_VP, C.c_uint64, _VP, C.c_uint64, C.POINTER(C.c_uint64)]),
    "ww_batch_run_noalloc": (C.c_int, [C.POINTER(Unit), C.c_uint32, _VP, _VP, _VP, C.c_uint32, _VP, _VP]),
    "ww_selftest_m2": (C.c_int, [C.c_int, C.c_uint64, _U64P, C.c_uint64, _U64P]),
    "ww_devtest_m2": (C.c_int, [C.c_int, C.c_int, C.c_uint64, _U64P, C.c_uint64, _U64P]),
    "ww_selftest_candidates": (C.c_int, [C.c_uint64, C.c_uint64, _U64P, C.c_uint64, C.POINTER(C.c_uint64),
                                         C.POINTER(C.c_uint64)]),
    "ww_random_primes": (C.c_int, [C.c_int, C.c_uint64, C.c_uint64, _U64P, C.POINTER(C.c_uint64)]),
    "ww_pipe_bench": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
}
for _name, (_res, _args) in _SIGS.items():
    _f = getattr(_L, _name)
    _f.restype = _res
    _f.argtypes = _args


def lib() -> C.CDLL:
    return _L


def check(rc: int, where: str) -> int:
    if rc < 0:
        raise WWError(rc, where)
    return rc


# ----------------------------------------------------------------- host helpers

def find_wheel_offset(start: int) -> tuple[int, int]:
    s = C.c_uint64(start)
    i = C.c_int32(0)
    check(_L.ww_find_wheel_offset(C.byref(s), C.byref(i)), "ww_find_wheel_offset")
    return int(s.value), int(i.value)


def is_prime(n: int) -> bool:
    return bool(_L.ww_is_prime(n))


def is_prp(n: int) -> bool:
    return bool(_L.ww_is_prp(n))


def parse_number(text: str) -> int:
    v = C.c_uint64(0)
    check(_L.ww_parse_number(text.encode(), C.byref(v)), f"ww_parse_number({text!r})")
    return int(v.value)


def format_hits(hits: list[tuple[int, int, int, int]]) -> tuple[str, int]:
    arr = (Hit * max(len(hits), 1))()
    for i, (p, r, rem, q) in enumerate(hits):
        arr[i].p, arr[i].result, arr[i].rem, arr[i].quot = p, r, rem, q
    buf = C.create_string_buffer(256 * max(len(hits), 1) + 1)
    dropped = C.c_uint32(0)
    check(_L.ww_format_hits(arr, len(hits), buf, len(buf), C.byref(dropped)), "ww_format_hits")
    return buf.value.decode(), int(dropped.value)


def state_write(file_a: str, file_b: str, start: int, stop: int, current: int, cksm: int, psum: float,
                pcnt: int, write_a_next: bool) -> bool:
    st = State(current, cksm, psum, pcnt, 0)
    a = C.c_int(1 if write_a_next else 0)
    check(_L.ww_state_write(file_a.encode(), file_b.encode(), start, stop, C.byref(st), C.byref(a)),
          "ww_state_write")
    return bool(a.value)


def state_read(file_a: str, file_b: str, start: int, stop: int):
    """(state dict, write_a_next) or None."""
    st = State()
    a = C.c_int(1)
    rc = check(_L.ww_state_read(file_a.encode(), file_b.encode(), start, stop, C.byref(st), C.byref(a)),
               "ww_state_read")
    if rc != 1:
        return None
    return dict(current=st.current, cksm=st.cksm, psum=st.psum, pcnt=st.pcnt), bool(a.value)


def prp_count_bound(lo: int, hi: int) -> int:
    return int(_L.ww_prp_count_bound(lo, hi))


def selftest_digits(primes: np.ndarray) -> np.ndarray:
    primes = np.ascontiguousarray(primes, dtype=np.uint64)
    out = np.zeros(4 * primes.size, dtype=np.uint64)
    check(_L.ww_selftest_digits(primes, primes.size, out), "ww_selftest_digits")
    return out.reshape(-1, 4)


def selftest_range(lo: int, hi: int) -> dict:
    a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint32()
    check(_L.ww_selftest_range(lo, hi, C.byref(a), C.byref(b), C.byref(c)), "ww_selftest_range")
    return dict(prp_count=a.value, checksum=b.value, result_count=c.value)


def selftest_m2(op: int, p: int, xy: np.ndarray) -> np.ndarray:
    xy = np.ascontiguousarray(xy, dtype=np.uint64).reshape(-1)
    n = xy.size // 4
    out = np.zeros(2 * n, dtype=np.uint64)
    check(_L.ww_selftest_m2(op, p, xy, n, out), "ww_selftest_m2")
    return out.reshape(-1, 2)


def devtest_m2(op: int, p: int, xy: np.ndarray, device: int = 0) -> np.ndarray:
    xy = np.ascontiguousarray(xy, dtype=np.uint64).reshape(-1)
    n = xy.size // 4
    out = np.zeros(2 * n, dtype=np.uint64)
    check(_L.ww_devtest_m2(device, op, p, xy, n, out), "ww_devtest_m2")
    return out.reshape(-1, 2)


def selftest_candidates(lo: int, hi: int) -> tuple[np.ndarray, int]:
    cap = (hi - lo) // 2 + 2
    out = np.zeros(cap, dtype=np.uint64)
    n, r = C.c_uint64(0), C.c_uint64(0)
    check(_L.ww_selftest_candidates(lo, hi, out, cap, C.byref(n), C.byref(r)), "ww_selftest_candidates")
    return out[: n.value], int(r.value)


def random_primes(seed: int, n: int, device: int = 0) -> tuple[np.ndarray, int]:
    out = np.zeros(n, dtype=np.uint64)
    used = C.c_uint64(0)
    check(_L.ww_random_primes(device, seed, n, out, C.byref(used)), "ww_random_primes")
    return out, int(used.value)


def pipe_bench(mode: int, device: int = 0) -> tuple[float, float]:
    ops, ms = C.c_double(0), C.c_double(0)
    check(_L.ww_pipe_bench(device, mode, C.byref(ops), C.byref(ms)), "ww_pipe_bench")
    return ops.value, ms.value


# -------------------------------------------------------------------- context

class Context:
    """Owns a ww_ctx: stream, PRP buffers, hit buffers, counters."""

    def __init__(self, device: int = 0, max_prps: int = 1 << 20, max_hits: int = 15000):
        h = C.c_void_p()
        check(_L.ww_open(device, C.byref(h)), "ww_open")
        self.h = h
        self.device = device
        self.reserve(max_prps, max_hits)

    def close(self) -> None:
        if self.h:
            _L.ww_close(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reserve(self, max_prps: int, max_hits: int = 15000) -> None:
        check(_L.ww_reserve(self.h, max_prps, max_hits), "ww_reserve")
        self.max_prps, self.max_hits = max_prps, max_hits

    def clear_results(self):
        check(_L.ww_clear_results(self.h), "ww_clear_results")

    def clear_segment(self):
        check(_L.ww_clear_segment(self.h), "ww_clear_segment")

    def sieve_prp(self, start: int, stop: int) -> None:
        """getsegprimes over [start, stop) after the wheel alignment of start
        (nothing to do when no number from start on is prime to 30, which
        happens only in the last few numbers below 2^64)."""
        s, i = C.c_uint64(start), C.c_int32(0)
        if _L.ww_find_wheel_offset(C.byref(s), C.byref(i)) != 0:
            return
        ks, idx = int(s.value), int(i.value)
        if ks >= stop:
            return
        check(_L.ww_sieve_prp(self.h, ks, stop, idx), "ww_sieve_prp")

    def set_sieve_depth(self, bits: int) -> None:
        """Deep primes below 2^bits in the sieve launches (20: per-segment primes only)."""
        check(_L.ww_set_sieve_depth(self.h, bits), "ww_set_sieve_depth")

    def sieve_depth(self) -> int:
        b = C.c_int(0)
        check(_L.ww_get_sieve_depth(self.h, C.byref(b)), "ww_get_sieve_depth")
        return b.value

    def deep_table(self, bits: int, first: int, n: int) -> tuple[np.ndarray, np.ndarray, int]:
        """Rows of the device's large-prime table: (r, ord_r(2), table length)."""
        r = np.zeros(max(n, 1), np.uint32)
        o = np.zeros(max(n, 1), np.uint32)
        tot = C.c_uint64(0)
        check(_L.ww_selftest_deep_table(self.h, bits, first, n, r.ctypes.data, o.ctypes.data, C.byref(tot)),
              "ww_selftest_deep_table")
        m = max(0, min(n, tot.value - first))
        return r[:m], o[:m], tot.value

    def set_sieve_shape(self, shape: int) -> None:
        """Sieve segments: 1 wide (2^20 numbers, 512 threads), 2 narrow (2^19, 256), 0 by width."""
        check(_L.ww_set_sieve_shape(self.h, shape), "ww_set_sieve_shape")

    def sieve_shape(self) -> int:
        v = C.c_int(0)
        check(_L.ww_get_sieve_shape(self.h, C.byref(v)), "ww_get_sieve_shape")
        return v.value

    def wieferich(self):
        check(_L.ww_wieferich(self.h), "ww_wieferich")

    def wallsunsun(self):
        check(_L.ww_wallsunsun(self.h), "ww_wallsunsun")

    def test_prps(self):
        check(_L.ww_test_prps(self.h), "ww_test_prps")

    def load_prps(self, primes: np.ndarray) -> None:
        primes = np.ascontiguousarray(primes, dtype=np.uint64)
        check(_L.ww_load_prps(self.h, primes.ctypes.data, primes.size), "ww_load_prps")

    def load_prps_ptr(self, host_ptr: int, n: int) -> None:
        check(_L.ww_load_prps(self.h, host_ptr, n), "ww_load_prps")

    def count_prps(self, lo: int, hi: int) -> int:
        """Exact PRP count of [lo, hi) from the sieve kernel (no list)."""
        n = C.c_uint64(0)
        check(_L.ww_count_prps(self.h, lo, hi, C.byref(n)), "ww_count_prps")
        return n.value

    def test_prps_host(self, primes: np.ndarray) -> None:
        """Both tests over a host list, copy and test pipelined in chunks."""
        primes = np.ascontiguousarray(primes, dtype=np.uint64)
        check(_L.ww_test_prps_host(self.h, primes.ctypes.data, primes.size), "ww_test_prps_host")
        self.sync()  # the pageable source must outlive the copies

    def test_prps_host_ptr(self, host_ptr: int, n: int) -> None:
        """As test_prps_host for a pinned host buffer; returns once queued."""
        check(_L.ww_test_prps_host(self.h, host_ptr, n), "ww_test_prps_host")

    def sync(self, timeout_ms: int = 600_000):
        check(_L.ww_sync(self.h, timeout_ms), "ww_sync")

    def marker(self, slot: int):
        check(_L.ww_marker(self.h, slot), "ww_marker")

    def wait_marker(self, slot: int, timeout_ms: int = 600_000):
        check(_L.ww_wait_marker(self.h, slot, timeout_ms), "ww_wait_marker")

    def elapsed_ms(self, a: int, b: int) -> float:
        ms = C.c_float(0)
        check(_L.ww_marker_elapsed(self.h, a, b, C.byref(ms)), "ww_marker_elapsed")
        return float(ms.value)

    def counters(self) -> dict:
        k = Counters()
        check(_L.ww_read_counters(self.h, C.byref(k)), "ww_read_counters")
        return dict(checksum=k.checksum, total_prp_count=k.total_prp_count, result_count=k.result_count,
                    seg_prp_count=k.seg_prp_count, max_prp_count=k.max_prp_count, overflow=k.overflow)

    def hits(self) -> list[tuple[int, int, int, int]]:
        cap = self.max_hits
        arr = (Hit * cap)()
        n = C.c_uint32(0)
        check(_L.ww_read_hits(self.h, arr, cap, C.byref(n)), "ww_read_hits")
        return [(arr[i].p, arr[i].result, arr[i].rem, arr[i].quot) for i in range(min(n.value, cap))]

    def prps(self) -> np.ndarray:
        cnt = self.counters()["seg_prp_count"]
        out = np.zeros(max(min(cnt, self.max_prps), 1), dtype=np.uint64)
        n = C.c_uint64(0)
        check(_L.ww_read_prps(self.h, out.ctypes.data, out.size, C.byref(n)), "ww_read_prps")
        return out[: min(n.value, out.size)]

    def buffers(self) -> Buffers:
        b = Buffers()
        check(_L.ww_get_buffers(self.h, C.byref(b)), "ww_get_buffers")
        return b

    # one-shot helpers ---------------------------------------------------
    def run_range(self, lo: int, hi: int, fused: bool = True, segment: int | None = None) -> dict:
        """Plain path over [lo, hi): clear, then per segment clearn -> sieve -> tests."""
        self.clear_results()
        seg = segment or hi - lo
        while seg > 1 and prp_count_bound(0, seg) > self.max_prps:  # keep every launch inside the buffer
            seg //= 2
        start = lo
        while start < hi:
            stop = min(start + seg, hi)
            self.clear_segment()
            self.sieve_prp(start, stop)
            if fused:
                self.test_prps()
            else:
                self.wieferich()
                self.wallsunsun()
            start = stop
        self.sync()
        c = self.counters()
        c["hits"] = [] if c["overflow"] & 2 else self.hits()
        return c


def batch_configs() -> list[tuple[int, int, int, int]]:
    n = C.c_uint32(0)
    check(_L.ww_batch_configs(None, 0, C.byref(n)), "ww_batch_configs")
    arr = (BatchCfg * n.value)()
    check(_L.ww_batch_configs(arr, n.value, C.byref(n)), "ww_batch_configs")
    return [c.as_tuple() for c in arr]


def _units(ranges) -> C.Array:
    arr = (Unit * max(len(ranges), 1))()
    for i, (a, b) in enumerate(ranges):
        arr[i].start, arr[i].end = a, b
    return arr


class Batch:
    """The batched search on a Context: many ranges in one persistent launch."""

    def __init__(self, ctx: Context, max_hits: int = 1 << 16):
        self.ctx = ctx
        check(_L.ww_batch_reserve_hits(ctx.h, max_hits), "ww_batch_reserve_hits")
        self.max_hits = max_hits

    def set_config(self, seg_words: int, threads: int, ppt: int, joint: int = 0) -> None:
        c = BatchCfg(seg_words, threads, ppt, joint)
        check(_L.ww_batch_set_config(self.ctx.h, C.byref(c)), "ww_batch_set_config")

    def config(self) -> tuple[int, int, int, int]:
        c = BatchCfg()
        check(_L.ww_batch_get_config(self.ctx.h, C.byref(c)), "ww_batch_get_config")
        return c.as_tuple()

    def tune(self, sample) -> tuple[tuple[int, int, int, int], float]:
        u = _units(sample)
        best = BatchCfg()
        ms = C.c_float(0)
        check(_L.ww_batch_tune(self.ctx.h, u, len(sample), C.byref(best), C.byref(ms)), "ww_batch_tune")
        return best.as_tuple(), float(ms.value)

    def submit(self, ranges) -> None:
        self._n = len(ranges)
        self._u = _units(ranges)
        check(_L.ww_batch_submit(self.ctx.h, self._u, self._n), "ww_batch_submit")

    def collect(self) -> list[dict]:
        """Per-range results.  When the hit records overflowed their buffer
        the results are still complete; hit_overflow is then True and
        hits() returns the records that fit."""
        out = (UnitResult * max(self._n, 1))()
        hc = C.c_uint32(0)
        rc = _L.ww_batch_collect(self.ctx.h, out, self._n, C.byref(hc))
        self.hit_overflow = rc == -4
        if rc != WW_OK and not self.hit_overflow:
            raise WWError(rc, "ww_batch_collect")
        self.hit_count = hc.value
        return [dict(checksum=r.checksum, prp_count=r.prp_count, hits=r.hits, tiles_done=r.tiles_done)
                for r in out[: self._n]]

    def run(self, ranges) -> list[dict]:
        self.submit(ranges)
        return self.collect()

    def hits(self) -> list[tuple[int, int, int, int, int]]:
        cap = self.max_hits
        arr = (Hit * cap)()
        units = (C.c_uint32 * cap)()
        n = C.c_uint32(0)
        rc = _L.ww_batch_hits(self.ctx.h, arr, units, cap, C.byref(n))
        if rc != WW_OK and rc != -4:  # -4: more hits than the buffer held; return those that fit
            raise WWError(rc, "ww_batch_hits")
        return [(units[i], arr[i].p, arr[i].result, arr[i].rem, arr[i].quot) for i in range(min(n.value, cap))]


class Server:
    """Continuous-batching request server on a Context."""

    def __init__(self, ctx: Context, prp_pool_bytes: int = 8 << 30, max_active: int = 64,
                 epoch_tiles: int = 0, max_hits: int = 1 << 15, store_prps: bool = True):
        self.ctx = ctx
        cfg = ServerCfg(prp_pool_bytes, max_active, epoch_tiles, max_hits, 1 if store_prps else 0)
        check(_L.ww_server_open(ctx.h, C.byref(cfg)), "ww_server_open")
        self.cap = max_active
        self._buf = (RequestResult * max_active)()

    def close(self):
        if self.ctx and self.ctx.h:
            _L.ww_server_close(self.ctx.h)
        self.ctx = None

    def submit(self, reqs) -> None:
        arr = (Request * max(len(reqs), 1))()
        for i, (rid, a, b) in enumerate(reqs):
            arr[i].id, arr[i].start, arr[i].end = rid, a, b
        check(_L.ww_server_submit(self.ctx.h, arr, len(reqs)), "ww_server_submit")

    def step(self) -> list[dict]:
        n = C.c_uint32(0)
        check(_L.ww_server_step(self.ctx.h, self._buf, self.cap, C.byref(n)), "ww_server_step")
        return [dict(id=r.id, checksum=r.checksum, prp_count=r.prp_count, prps_stored=r.prps_stored,
                     hits=r.hits, status=r.status, t_submit=r.t_submit, t_admit=r.t_admit, t_done=r.t_done)
                for r in self._buf[: n.value]]

    def status(self) -> tuple[int, int, int]:
        q, a, u = C.c_uint32(0), C.c_uint32(0), C.c_uint64(0)
        check(_L.ww_server_status(self.ctx.h, C.byref(q), C.byref(a), C.byref(u)), "ww_server_status")
        return q.value, a.value, u.value

    def hits(self, rid: int) -> list[tuple[int, int, int, int]]:
        cap = 4096
        arr = (Hit * cap)()
        n = C.c_uint32(0)
        check(_L.ww_server_hits(self.ctx.h, rid, arr, cap, C.byref(n)), "ww_server_hits")
        return [(arr[i].p, arr[i].result, arr[i].rem, arr[i].quot) for i in range(min(n.value, cap))]

    def prps(self, rid: int, cap: int) -> np.ndarray:
        out = np.zeros(max(cap, 1), dtype=np.uint64)
        n = C.c_uint64(0)
        check(_L.ww_server_prps(self.ctx.h, rid, out.ctypes.data, cap, C.byref(n)), "ww_server_prps")
        return out[: min(n.value, cap)]

    def drain(self, max_steps: int = 100000) -> list[dict]:
        done = []
        for _ in range(max_steps):
            done += self.step()
            q, a, _ = self.status()
            if q == 0 and a == 0:
                break
        return done


def uneven_units(seed: int, n: int, wmin: float = 1e6, wmax: float = 1e10, smin: int = 10**15,
                 smax: int = 2**64 - 10**10, align: int = 30) -> list[tuple[int, int]]:
    """The uneven-range mix: widths log-uniform in [wmin, wmax], starts
    uniform in [smin, smax] rounded down to multiples of `align`."""
    rng = np.random.default_rng(seed)
    widths = np.exp(rng.uniform(np.log(wmin), np.log(wmax), n)).astype(np.float64)
    starts = rng.integers(smin // align, smax // align, n, dtype=np.uint64, endpoint=False)
    out = []
    for s, w in zip(starts, widths):
        a = int(s) * align
        out.append((a, a + int(w)))
    return out


def digits(primes: np.ndarray, device: int = 0) -> np.ndarray:
    """Per-prime (s0, s1, c20, c21) on the GPU via ww_launch_digits (torch for device memory)."""
    import torch

    primes = np.ascontiguousarray(primes, dtype=np.uint64)
    dev = torch.device("cuda", device)
    p = torch.from_numpy(primes.view(np.int64)).to(dev)
    out = torch.empty(4 * primes.size, dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    check(_L.ww_launch_digits(p.data_ptr(), primes.size, out.data_ptr(), stream), "ww_launch_digits")
    torch.cuda.synchronize(dev)
    return out.cpu().numpy().view(np.uint64).reshape(-1, 4)


def exported_symbols() -> list[str]:
    return sorted(_SIGS)


def header_symbols(header: Path | None = None) -> list[str]:
    import re

    header = header or PKG.parent / "include" / "wwcuda.h"
    text = header.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ww_[a-z0-9_]+)\s*\(", text)))


if os.environ.get("WW_DEBUG_IMPORT"):
    print("libwwcuda loaded from", LIB_PATH)
