"""Small helpers shared by the tests."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from diffuse_vs_gfm_mms_b200 import abi

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def desc_from_array(a: np.ndarray) -> abi.Desc:
    """Descriptor from stored bytes; fields added after the fixture was
    written (at the end of the struct) keep their zero default."""
    d = abi.Desc()
    raw = a.tobytes()
    C.memmove(C.byref(d), raw, min(len(raw), C.sizeof(abi.Desc)))
    return d


def bitwise_equal(a, b) -> bool:
    """Equal bit for bit, except that NaN == NaN (both fields must agree on NaNs)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return a.shape == b.shape and bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))


def ndiff(a, b) -> int:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return int(np.sum(~((a == b) | (np.isnan(a) & np.isnan(b)))))


def rel_l1(test: np.ndarray, ref: np.ndarray) -> np.ndarray:
    """Relative L1 per conserved variable: sum|test-ref| / sum|ref| (the cell
    volume cancels; src/graphing/error_metrics.py:76-85 defines the L1)."""
    test = np.asarray(test).reshape(ref.shape[0], -1)
    ref = np.asarray(ref).reshape(ref.shape[0], -1)
    den = np.abs(ref).sum(axis=1)
    den = np.where(den > 0, den, 1.0)
    return np.abs(test - ref).sum(axis=1) / den


def load(name: str):
    return np.load(os.path.join(GOLDEN, name))
