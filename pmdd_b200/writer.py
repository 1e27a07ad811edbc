"""Frontier CSV.gz and stats JSONL output over libpmdd_host.so's writers.

`write_frontier_csv_gz` writes one file now; `FrontierWriter` queues results to a pool
of writer threads so that a serving loop hands each one over and goes on (the
reference writes from the enumerating thread through a `gzip -c` child per file,
src/pmdd/util/output_utils.cpp:87-152).  The decompressed CSV is the reference's text:
points sorted ascending lexicographically, one per line, objectives joined by ','.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _native


def _points(points) -> tuple:
    pts = np.asarray(points)
    if pts.ndim != 2:
        raise ValueError("points must be a (num_points, nobjs) array")
    if pts.dtype == np.int64 or pts.dtype == np.uint64:
        pts = np.ascontiguousarray(pts, dtype=np.int64)
        elem = 8
    else:
        pts = np.ascontiguousarray(pts, dtype=np.int32)
        elem = 4
    return pts, elem


def write_frontier_csv_gz(points, path: str, sort: bool = True) -> None:
    pts, elem = _points(points)
    err = ctypes.create_string_buffer(512)
    rc = _native.host_lib().pmdd_write_frontier_csv_gz(pts.ctypes.data, pts.shape[0], pts.shape[1], elem,
                                                        1 if sort else 0, path.encode(), err, len(err))
    if rc != _native.PMDD_OK:
        raise OSError(f"{_native.STATUS_NAMES.get(rc, rc)}: {err.value.decode(errors='replace')}")


class FrontierWriter:
    """Asynchronous writer; `submit` copies the points and returns at once."""

    def __init__(self, threads: int = 0):
        err = ctypes.create_string_buffer(512)
        self._lib = _native.host_lib()
        self._h = self._lib.pmdd_writer_create(int(threads), err, len(err))
        if not self._h:
            raise ValueError(err.value.decode(errors="replace"))

    def submit(self, points, csv_gz_path: Optional[str] = None, jsonl_path: Optional[str] = None,
               record: Optional[str] = None) -> None:
        pts, elem = _points(points) if points is not None else (np.zeros((0, 1), dtype=np.int32), 4)
        rc = self._lib.pmdd_writer_submit(self._h, pts.ctypes.data, pts.shape[0], pts.shape[1], elem,
                                          csv_gz_path.encode() if csv_gz_path else None,
                                          jsonl_path.encode() if jsonl_path else None,
                                          record.encode() if record is not None else None)
        if rc != _native.PMDD_OK:
            raise ValueError("writer rejected the result (no output path, a record with a newline, or bad points)")

    def pending(self) -> int:
        return int(self._lib.pmdd_writer_pending(self._h))

    def flush(self) -> int:
        """Waits for the queue; returns how many results were written since the last
        flush and raises if any failed."""
        written = ctypes.c_int64(0)
        err = ctypes.create_string_buffer(512)
        failed = self._lib.pmdd_writer_flush(self._h, ctypes.byref(written), err, len(err))
        if failed:
            raise OSError(f"{failed} result(s) not written: {err.value.decode(errors='replace')}")
        return int(written.value)

    def close(self) -> None:
        if self._h:
            self._lib.pmdd_writer_destroy(self._h)
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
