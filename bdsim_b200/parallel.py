"""Map over independent work items with per-item failure capture
(python/bdsim/parallel.py of the bdsim project).

The ensemble layer batches trajectories onto the GPU itself (backend="cuda");
`parallel_map` remains for user code that maps arbitrary functions.
"""


class Failure:
    """Stands in for the result of an item whose function raised."""

    __slots__ = ("index", "error")

    def __init__(self, index, error):
        self.index = index
        self.error = error

    def __repr__(self):
        return f"Failure(index={self.index}, error={self.error!r})"

    @property
    def message(self):
        return f"{type(self.error).__name__}: {self.error}"


class _Guarded:
    __slots__ = ("fn",)

    def __init__(self, fn):
        self.fn = fn

    def __call__(self, item):
        try:
            return self.fn(item)
        except Exception as exc:
            return Failure(None, exc)


def parallel_map(fn, items, *, backend="serial", n_workers=None, on_error="raise"):
    """fn over items in order; backend "serial" or "processes";
    on_error="skip" returns Failure objects in place of raised items."""
    items = list(items)
    if on_error not in ("raise", "skip"):
        raise ValueError(f"on_error must be 'raise' or 'skip', got {on_error!r}")
    call = fn if on_error == "raise" else _Guarded(fn)
    if backend == "serial":
        out = [call(x) for x in items]
    elif backend == "processes":
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        with ProcessPoolExecutor(max_workers=n_workers, mp_context=mp.get_context("spawn")) as ex:
            out = list(ex.map(call, items))
    else:
        raise ValueError(f"unknown backend {backend!r} (use 'serial' or 'processes')")
    for i, r in enumerate(out):
        if isinstance(r, Failure):
            r.index = i
    return out
