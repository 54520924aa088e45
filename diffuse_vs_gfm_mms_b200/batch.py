"""Batched DIM solves: many independent grids advanced together on one GPU.

``Batch`` wraps the dimgpu_batch_* C-ABI: instances of one material count
and dimension, each with its own grid, materials, cfl, dt_max and step
budget, advance together through persistent-grid launches replayed from a
captured CUDA graph.  An instance's result is bit-identical to running the
same grid alone through ``Session``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .abi import Desc, dptr
from .native import DimGpuError, lib


class Batch:
    def __init__(self, nmat: int, dim: int):
        h = C.c_void_p()
        self._check(lib().dimgpu_batch_create(nmat, dim, C.byref(h)), None)
        self._h = h
        self.nmat, self.dim = nmat, dim
        self.descs: dict[int, Desc] = {}

    def _check(self, rc, h=...):
        if rc != 0:
            handle = self._h if h is ... else h
            msg = lib().dimgpu_batch_last_error(handle) if handle else lib().dimgpu_last_error(None)
            raise DimGpuError(rc, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "_h", None):
            lib().dimgpu_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, desc: Desc, U: np.ndarray, steps: int, cfl: float, dt_max: float = 1e300) -> int:
        U = np.ascontiguousarray(U, dtype=np.float64)
        i = C.c_int()
        self._check(lib().dimgpu_batch_add(self._h, C.byref(desc), dptr(U), steps, cfl, dt_max, C.byref(i)))
        self.descs[i.value] = desc.copy()
        return i.value

    def remove(self, iid: int) -> None:
        self._check(lib().dimgpu_batch_remove(self._h, iid))
        self.descs.pop(iid, None)

    def run(self, n: int) -> None:
        self._check(lib().dimgpu_batch_run(self._h, n))

    def status(self, iid: int) -> tuple[int, int]:
        done, left = C.c_int(), C.c_int()
        self._check(lib().dimgpu_batch_status(self._h, iid, C.byref(done), C.byref(left)))
        return done.value, left.value

    def download(self, iid: int, with_dts: bool = True):
        d = self.descs[iid]
        out = np.empty((d.nvar, d.ncell))
        done, _ = self.status(iid)
        dts = np.zeros(max(done, 1))
        self._check(lib().dimgpu_batch_download(self._h, iid, dptr(out), out.size, dptr(dts) if with_dts else None))
        return out, dts[:done]

    def reserve(self, max_cells: int, max_instances: int, max_steps: int) -> None:
        """Arena mode: device memory for every later add is reserved now, so
        add / remove allocate and synchronise nothing."""
        self._check(lib().dimgpu_batch_reserve(self._h, max_cells, max_instances, max_steps))

    def arena_used(self) -> tuple[int, int]:
        cells, dts = C.c_longlong(), C.c_longlong()
        self._check(lib().dimgpu_batch_arena_used(self._h, C.byref(cells), C.byref(dts)))
        return cells.value, dts.value

    def enqueue(self, n: int) -> None:
        """Enqueue up to n steps without waiting (see wait)."""
        self._check(lib().dimgpu_batch_enqueue(self._h, n))

    def wait(self) -> None:
        self._check(lib().dimgpu_batch_wait(self._h))

    def set_stream(self, stream_handle: int | None) -> None:
        self._check(lib().dimgpu_batch_set_stream(self._h, C.c_void_p(stream_handle or 0)))

    def set_grid(self, ctas: int) -> None:
        self._check(lib().dimgpu_batch_set_grid(self._h, ctas))

    def __len__(self):
        return int(lib().dimgpu_batch_size(self._h))
