"""Many SCFT instances of several grid shapes solved together.

One engine per grid shape (each owns its CUDA stream); the engines are
driven concurrently from host threads (the C ABI calls release the GIL),
so the lamellar, cylinder and sphere batches of a mixed workload overlap on
the GPU instead of running one after another.
"""
from __future__ import annotations

import threading
from typing import List, Optional, Sequence

import numpy as np

from .engine import Engine, FP64


class ShapeBatch:
    def __init__(self, systems, omega0, group: Optional[str] = None, precision: int = FP64):
        self.systems = list(systems)
        self.omega0 = np.asarray(omega0)
        self.group = group
        self.engine = Engine(self.systems, precision)
        if group:
            for i in range(len(self.systems)):
                self.engine.set_symmetry(i, group)
        self.result = None
        self.error = None


def solve_batches(batches: Sequence[ShapeBatch], **am_kwargs) -> List[list]:
    """Anderson solves of every batch concurrently; returns the per-instance
    result dicts of each batch (pscfg_iterate_am)."""
    def run(b: ShapeBatch):
        try:
            _, _, b.result = b.engine.iterate_am(b.omega0, **am_kwargs)
        except Exception as exc:  # reported after the join
            b.error = exc

    threads = [threading.Thread(target=run, args=(b,)) for b in batches]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for b in batches:
        if b.error is not None:
            raise b.error
    return [b.result for b in batches]
