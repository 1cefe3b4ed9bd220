"""Bitwise comparison of state arrays for the parity tests (0 ulp).

Two arrays match when their bytes are equal, with one allowance: a 32-bit word that is a NaN on both sides matches
whatever its payload. The reference's EPA can return a NaN witness point when a car's box lands flat on the floor (a
degenerate polytope face), and the car then carries NaN from that tick on in the reference and in this build alike;
x86 produces the NaN 0xffc00000 where the GPU produces 0x7fffffff, so only the payload differs. Every other bit,
including which words are NaN and on which tick they became NaN, must match.
"""
from __future__ import annotations

import numpy as np


def _words(a: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    flat = np.ascontiguousarray(a).reshape(-1)
    n = (flat.size // 4) * 4
    return flat[:n].view(np.uint32), flat[n:]


def mismatched_bytes(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Byte offsets (into the flattened arrays) that differ, NaN words on both sides excepted."""
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    assert a.shape == b.shape and a.dtype == np.uint8 and b.dtype == np.uint8
    if np.array_equal(a, b):
        return np.zeros(0, np.int64)
    wa, ta = _words(a)
    wb, tb = _words(b)
    fa, fb = wa.view(np.float32), wb.view(np.float32)
    bad_words = (wa != wb) & ~(np.isnan(fa) & np.isnan(fb))
    bad = np.repeat(bad_words, 4) & (a.reshape(-1)[: wa.size * 4] != b.reshape(-1)[: wb.size * 4])
    tail = np.nonzero(ta != tb)[0] + wa.size * 4
    return np.concatenate([np.nonzero(bad)[0], tail])


def equal(a: np.ndarray, b: np.ndarray) -> bool:
    return mismatched_bytes(a, b).size == 0


def first_mismatch(pairs, row_bytes: dict[str, int] | None = None):
    """pairs: iterable of (label, oracle_array, gpu_array). Returns a description of the first mismatch, or None."""
    for label, a, b in pairs:
        d = mismatched_bytes(a, b)
        if d.size:
            width = (row_bytes or {}).get(label)
            where = f"rows {sorted(set((d // width).tolist()))[:8]} bytes {sorted(set((d % width).tolist()))[:16]}" \
                if width else f"bytes {d[:16].tolist()}"
            return f"{label}: {where}"
    return None
