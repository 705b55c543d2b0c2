"""Test-side binding of the oracle (oracle/liboracle.so) and of the reference's
own CPU counter built into oracle/_ref.  Checker only: nothing in the product
imports this module."""
from __future__ import annotations

import ctypes
import os
import re
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
GGCOUNT = os.path.join(ROOT, "oracle", "_ref", "ggcount_multi")
REFERENCE_ROOT_FILE = os.path.join(ROOT, "oracle", "_ref", "reference_root")


def reference_root():
    """The reference tree, for CPU tests that import its own Python tools:
    ONEESAN_REFERENCE_ROOT if set, else the tree `make -C oracle ref
    REF_ROOT=...` built oracle/_ref from; None when neither is present."""
    root = os.environ.get("ONEESAN_REFERENCE_ROOT")
    if not root and os.path.exists(REFERENCE_ROOT_FILE):
        with open(REFERENCE_ROOT_FILE) as f:
            root = f.read().strip()
    return root if root and os.path.isdir(root) else None

# The first 48 primes below 2^32 in descending order: the reference's CRT prime
# table (scripts/solve/path_bound.py:5-18) is exactly this sequence.
def largest_primes_below_2_32(count: int) -> list[int]:
    out, x = [], (1 << 32) - 1
    while len(out) < count:
        if _is_prime(x):
            out.append(x)
        x -= 1
    return out


def _is_prime(x: int) -> bool:
    if x < 2:
        return False
    for q in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        if x % q == 0:
            return x == q
    d, s = x - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in (2, 3, 5, 7, 11, 13, 17):
        y = pow(a, d, x)
        if y in (1, x - 1):
            continue
        for _ in range(s - 1):
            y = y * y % x
            if y == x - 1:
                break
        else:
            return False
    return True


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "lib"], check=True,
                           stdout=subprocess.DEVNULL)
        L = ctypes.CDLL(ORACLE_SO)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        L.oracle_hdp.argtypes = [ctypes.c_int, ctypes.c_int]
        L.oracle_hdp.restype = ctypes.c_uint64
        L.oracle_rank.argtypes = [ctypes.c_uint64, ctypes.c_int]
        L.oracle_rank.restype = ctypes.c_uint64
        L.oracle_unrank.argtypes = [ctypes.c_uint64, ctypes.c_int]
        L.oracle_unrank.restype = ctypes.c_uint64
        L.oracle_main_states.argtypes = [ctypes.c_int]
        L.oracle_main_states.restype = ctypes.c_uint64
        L.oracle_include.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_uint64)]
        L.oracle_forward_cell.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_uint32, u32p, u32p, u32p, u32p]
        L.oracle_residue.argtypes = [ctypes.c_int, ctypes.c_uint32, u32p]
        L.oracle_dfs_count.argtypes = [ctypes.c_int, ctypes.c_int]
        L.oracle_dfs_count.restype = ctypes.c_uint64
        L.oracle_first_row_state.argtypes = [ctypes.c_uint64, ctypes.c_int]
        L.oracle_first_row_state.restype = ctypes.c_uint64
        _lib = L
    return _lib


def main_states(width: int) -> int:
    return int(lib().oracle_main_states(width))


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def forward_cell(width: int, p: int, mod: int, main: np.ndarray, block: np.ndarray):
    main = np.ascontiguousarray(main, dtype=np.uint32)
    block = np.ascontiguousarray(block, dtype=np.uint32)
    mo = np.empty_like(main)
    bo = np.empty_like(block)
    rc = lib().oracle_forward_cell(width, p, mod, _ptr(main), _ptr(block), _ptr(mo), _ptr(bo))
    assert rc == 0
    return mo, bo


def residue(n: int, mod: int) -> int:
    out = ctypes.c_uint32()
    assert lib().oracle_residue(n, mod, ctypes.byref(out)) == 0
    return int(out.value)


def dfs_count(n: int, threads: int | None = None) -> int:
    return int(lib().oracle_dfs_count(n, threads or os.cpu_count() or 1))


def include(word: int, width: int, p: int):
    out = ctypes.c_uint64()
    kind = lib().oracle_include(word, width, p, ctypes.byref(out))
    return kind, int(out.value)


def rank(word: int, width: int) -> int:
    return int(lib().oracle_rank(word, width))


def unrank(r: int, width: int) -> int:
    return int(lib().oracle_unrank(r, width))


def ggcount_available() -> bool:
    return os.path.exists(GGCOUNT)


def ggcount_residue(n: int, mod: int, threads: int | None = None) -> int:
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    out = subprocess.run([GGCOUNT, "-q", str(n), f"%{mod}"], check=True, capture_output=True, text=True,
                         env=env).stdout
    m = re.match(r"\s*(\d+)", out)
    assert m, out
    return int(m.group(1))


def crt(residues: dict[int, int]) -> tuple[int, int]:
    x, m = 0, 1
    for p, r in residues.items():
        t = ((r - x) * pow(m, -1, p)) % p
        x += m * t
        m *= p
    return x, m
