"""Per-trajectory failures of a batched ensemble.

On the device every chain carries a status word; a chain whose status has a
fatal bit (not positive definite, rtsafe failure, non-finite positions, bad
parameter) stops while the rest of its launch continues. The run layer reports
such a chain as a `Failure` in its result slot, the object bdsim's own
`_drop_failures` / `MAX_FAILED_FRACTION` logic recognises
(python/bdsim/ensemble.py:244-263 of the bdsim project): it exposes the
trajectory's position (`index`), the exception (`error`) and a one-line
`message`. There is no process pool here: trajectories are batched onto the GPU
rather than mapped over host processes.
"""
from __future__ import annotations

from dataclasses import dataclass


@dataclass(eq=False)
class Failure:
    """Result slot of a trajectory that stopped on a fatal status."""

    index: int | None
    error: BaseException

    @property
    def message(self) -> str:
        return f"{type(self.error).__name__}: {self.error}"
