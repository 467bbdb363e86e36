"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU checker.

`Oracle` wraps liboracle.so (the C restatement in ww_oracle.c); `RefCPU`
wraps _ref/libwwref.so (the reference's own wwcpu.cpp + prime.h compiled in
place).  Only the tests, the smoke check and the benchmark's CPU-baseline
leg import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


class WoDigits(C.Structure):
    _fields_ = [("d0", C.c_uint64), ("d1", C.c_uint64)]


class WoHit(C.Structure):
    _fields_ = [("p", C.c_uint64), ("result", C.c_int32), ("rem", C.c_int32),
                ("quot", C.c_int32), ("pad", C.c_int32)]


class WoSummary(C.Structure):
    _fields_ = [("prp_count", C.c_uint64), ("checksum", C.c_uint64),
                ("cpu_results", C.c_uint64), ("gpu_results", C.c_uint64)]


_U64P = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_U32P = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_I32P = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def _nthreads() -> int:
    return max(1, os.cpu_count() or 1)


class Oracle:
    def __init__(self, path: Path | None = None):
        path = path or HERE / "liboracle.so"
        if not path.exists():
            build()
        L = C.CDLL(str(path))
        self.L = L
        L.wo_sprp2.argtypes = [C.c_uint64]
        L.wo_small_factor.argtypes = [C.c_uint64]
        L.wo_is_prp.argtypes = [C.c_uint64]
        L.wo_is_prime.argtypes = [C.c_uint64]
        L.wo_inv64.argtypes = [C.c_uint64]
        L.wo_inv64.restype = C.c_uint64
        L.wo_wieferich_digits.argtypes = [C.c_uint64]
        L.wo_wieferich_digits.restype = WoDigits
        L.wo_wss_digits.argtypes = [C.c_uint64]
        L.wo_wss_digits.restype = WoDigits
        L.wo_find_wheel_offset.argtypes = [C.POINTER(C.c_uint64), C.POINTER(C.c_int32)]
        L.wo_scan_range.argtypes = [C.c_uint64, C.c_uint64, C.c_int, C.POINTER(WoSummary),
                                    C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64]
        L.wo_test_list.argtypes = [_U64P, C.c_uint64, C.c_int, C.POINTER(WoSummary),
                                   C.c_void_p, C.c_uint64]
        L.wo_list_digits.argtypes = [_U64P, C.c_uint64, C.c_int, C.c_void_p, C.c_void_p]
        L.wo_format_results.argtypes = [C.POINTER(WoHit), C.c_uint64, C.c_char_p, C.c_size_t,
                                        C.POINTER(C.c_uint32)]
        L.wo_parse_number.argtypes = [C.c_char_p, C.POINTER(C.c_uint64)]
        L.wo_splitmix64.argtypes = [C.c_uint64, C.c_uint64]
        L.wo_splitmix64.restype = C.c_uint64
        L.wo_random_primes.argtypes = [C.c_uint64, C.c_uint64, _U64P, C.c_int]
        L.wo_random_primes.restype = C.c_uint64

    # scalar helpers -----------------------------------------------------
    def sprp2(self, n: int) -> bool:
        return bool(self.L.wo_sprp2(n))

    def small_factor(self, n: int) -> bool:
        return bool(self.L.wo_small_factor(n))

    def is_prp(self, n: int) -> bool:
        return bool(self.L.wo_is_prp(n))

    def is_prime(self, n: int) -> bool:
        return bool(self.L.wo_is_prime(n))

    def inv64(self, p: int) -> int:
        return int(self.L.wo_inv64(p))

    def wieferich_digits(self, p: int) -> tuple[int, int]:
        d = self.L.wo_wieferich_digits(p)
        return int(d.d0), int(d.d1)

    def wss_digits(self, p: int) -> tuple[int, int]:
        d = self.L.wo_wss_digits(p)
        return int(d.d0), int(d.d1)

    def wheel_offset(self, start: int) -> tuple[int, int]:
        s = C.c_uint64(start)
        i = C.c_int32(0)
        self.L.wo_find_wheel_offset(C.byref(s), C.byref(i))
        return int(s.value), int(i.value)

    def parse_number(self, text: str) -> tuple[int, int]:
        v = C.c_uint64(0)
        rc = self.L.wo_parse_number(text.encode(), C.byref(v))
        return int(rc), int(v.value)

    # bulk helpers -------------------------------------------------------
    def scan_range(self, lo: int, hi: int, nthreads: int | None = None, want_prps: bool = False,
                   prp_cap: int = 0, hit_cap: int = 4096):
        """Returns (summary dict, prps ndarray|None, hits list)."""
        s = WoSummary()
        prps = None
        pptr = None
        if want_prps:
            prps = np.zeros(max(prp_cap, 1), dtype=np.uint64)
            pptr = prps.ctypes.data
        hits = (WoHit * max(hit_cap, 1))()
        self.L.wo_scan_range(lo, hi, nthreads or _nthreads(), C.byref(s), pptr, prp_cap,
                             C.cast(hits, C.c_void_p), hit_cap)
        summ = dict(prp_count=s.prp_count, checksum=s.checksum, cpu_results=s.cpu_results,
                    gpu_results=s.gpu_results)
        nh = min(s.gpu_results, hit_cap)
        hl = [(h.p, h.result, h.rem, h.quot) for h in hits[:nh]]
        if prps is not None:
            prps = np.sort(prps[: min(s.prp_count, prp_cap)])
        return summ, prps, hl

    def test_list(self, primes: np.ndarray, nthreads: int | None = None, hit_cap: int = 4096):
        primes = np.ascontiguousarray(primes, dtype=np.uint64)
        s = WoSummary()
        hits = (WoHit * max(hit_cap, 1))()
        self.L.wo_test_list(primes, primes.size, nthreads or _nthreads(), C.byref(s),
                            C.cast(hits, C.c_void_p), hit_cap)
        nh = min(s.gpu_results, hit_cap)
        return (dict(prp_count=s.prp_count, checksum=s.checksum, cpu_results=s.cpu_results,
                     gpu_results=s.gpu_results),
                [(h.p, h.result, h.rem, h.quot) for h in hits[:nh]])

    def list_digits(self, primes: np.ndarray, nthreads: int | None = None):
        """(N, 2) arrays of Wieferich digits and WSS digits."""
        primes = np.ascontiguousarray(primes, dtype=np.uint64)
        w = np.zeros((primes.size, 2), dtype=np.uint64)
        s = np.zeros((primes.size, 2), dtype=np.uint64)
        self.L.wo_list_digits(primes, primes.size, nthreads or _nthreads(), w.ctypes.data, s.ctypes.data)
        return w, s

    def format_results(self, hits: list[tuple[int, int, int, int]]) -> tuple[int, str, int]:
        arr = (WoHit * max(len(hits), 1))()
        for i, (p, r, rem, q) in enumerate(hits):
            arr[i].p, arr[i].result, arr[i].rem, arr[i].quot = p, r, rem, q
        buf = C.create_string_buffer(256 * max(len(hits), 1) + 1)
        dropped = C.c_uint32(0)
        rc = self.L.wo_format_results(arr, len(hits), buf, len(buf), C.byref(dropped))
        return int(rc), buf.value.decode(), int(dropped.value)

    def random_primes(self, seed: int, n: int, nthreads: int | None = None) -> tuple[np.ndarray, int]:
        out = np.zeros(n, dtype=np.uint64)
        used = self.L.wo_random_primes(seed, n, out, nthreads or _nthreads())
        return out, int(used)

    def splitmix64(self, seed: int, i: int) -> int:
        return int(self.L.wo_splitmix64(seed, i))


class RefCPU:
    """The reference's own CPU path (wwcpu.cpp, prime.h) compiled in place."""

    def __init__(self, path: Path | None = None):
        path = path or HERE / "_ref" / "libwwref.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (oracle/Makefile needs the reference tree)")
        L = C.CDLL(str(path))
        self.L = L
        L.ref_wieferich.argtypes = [C.c_uint64, C.POINTER(C.c_uint64)]
        L.ref_wallsunsun.argtypes = [C.c_uint64, C.POINTER(C.c_uint64)]
        L.ref_is_prp.argtypes = [C.c_uint64]
        L.ref_list_terms.argtypes = [_U64P, C.c_uint64, _U32P, _U32P, _I32P, _I32P]
        L.ref_prp_list.argtypes = [C.c_uint64, C.c_uint64, _U64P, C.c_uint64]
        L.ref_prp_list.restype = C.c_uint64
        L.ref_scan_range.argtypes = [C.c_uint64, C.c_uint64, C.c_int, C.POINTER(C.c_uint64),
                                     C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.ref_test_list.argtypes = [_U64P, C.c_uint64, C.c_int, C.POINTER(C.c_uint64),
                                    C.POINTER(C.c_uint64)]

    @staticmethod
    def available(path: Path | None = None) -> bool:
        return (path or HERE / "_ref" / "libwwref.so").exists()

    def list_terms(self, primes: np.ndarray):
        primes = np.ascontiguousarray(primes, dtype=np.uint64)
        n = primes.size
        wt = np.zeros(n, np.uint32)
        st = np.zeros(n, np.uint32)
        wh = np.zeros(n, np.int32)
        sh = np.zeros(n, np.int32)
        self.L.ref_list_terms(primes, n, wt, st, wh, sh)
        return wt, st, wh, sh

    def prp_list(self, lo: int, hi: int, cap: int) -> np.ndarray:
        out = np.zeros(max(cap, 1), np.uint64)
        k = self.L.ref_prp_list(lo, hi, out, cap)
        return out[: min(k, cap)]

    def scan_range(self, lo: int, hi: int, nthreads: int | None = None):
        a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        self.L.ref_scan_range(lo, hi, nthreads or _nthreads(), C.byref(a), C.byref(b), C.byref(c))
        return dict(prp_count=a.value, checksum=b.value, cpu_results=c.value)

    def test_list(self, primes: np.ndarray, nthreads: int | None = None):
        primes = np.ascontiguousarray(primes, dtype=np.uint64)
        b, c = C.c_uint64(), C.c_uint64()
        self.L.ref_test_list(primes, primes.size, nthreads or _nthreads(), C.byref(b), C.byref(c))
        return dict(checksum=b.value, cpu_results=c.value)
