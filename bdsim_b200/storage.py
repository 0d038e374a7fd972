"""Trajectory storage with the layout of bdsim's run directories
(python/bdsim/storage.py of the bdsim project):

    run_dir/manifest.json, run_dir/traj_NNNNN.<ext>

Each trajectory file holds `step` (n_snap,), `time` (n_snap,), `positions`
(n_snap, N, 3), optional `forces` (n_snap, N, 3) and scalar attributes. The
container is HDF5 (.h5, gzip) when h5py is importable, otherwise a NumPy .npz
archive with the same dataset names (h5py is not part of every image).

`RunWriter` takes a run's snapshots chunk by chunk as they come off the GPU
(copied into pinned host buffers on the launch stream, each followed by an
event) and spools them to disk on a background thread while the device runs
the next chunk; at the end it writes one file per trajectory from the spool.
Host memory holds at most `max_pending` snapshots, not the whole run.
`SnapshotSink` writes whole trajectories on a background thread.
h5py is not installed in every image (not in this one): the fallback is .npz.
"""
from __future__ import annotations

import json
import os
import queue
import threading

import numpy as np


def _have_h5py() -> bool:
    try:
        import h5py  # noqa: F401
        return True
    except ImportError:
        return False


def trajectory_path(directory, index, ext=None):
    ext = ext or ("h5" if _have_h5py() else "npz")
    return os.path.join(directory, f"traj_{index:05d}.{ext}")


def write_trajectory(path, steps, times, positions, forces=None, attrs=None, compression="gzip"):
    """Write one trajectory's snapshots to `path` (.h5 or .npz)."""
    steps = np.asarray(steps)
    times = np.asarray(times, dtype=np.float64)
    positions = np.asarray(positions, dtype=np.float64)
    attrs = dict(attrs or {})
    attrs["has_forces"] = forces is not None
    if path.endswith(".h5"):
        import h5py
        with h5py.File(path, "w") as f:
            for k, v in attrs.items():
                f.attrs[k] = v
            f.create_dataset("step", data=steps)
            f.create_dataset("time", data=times)
            f.create_dataset("positions", data=positions, compression=compression)
            if forces is not None:
                f.create_dataset("forces", data=np.asarray(forces, dtype=np.float64), compression=compression)
    else:
        data = {"step": steps, "time": times, "positions": positions, "attrs": np.array(json.dumps(attrs))}
        if forces is not None:
            data["forces"] = np.asarray(forces, dtype=np.float64)
        with open(path, "wb") as fh:
            np.savez_compressed(fh, **data)


def write_manifest(directory, manifest):
    os.makedirs(directory, exist_ok=True)
    with open(os.path.join(directory, "manifest.json"), "w") as fh:
        json.dump(manifest, fh, indent=2, default=str)


class Trajectory:
    """Lazy reader for one trajectory file; iterating yields (step, time, R, F_or_None)."""

    def __init__(self, path):
        self.path = path

    def _load(self):
        if self.path.endswith(".h5"):
            import h5py
            with h5py.File(self.path, "r") as f:
                d = {k: f[k][()] for k in f.keys()}
                d["attrs"] = dict(f.attrs)
            return d
        with np.load(self.path) as z:
            d = {k: z[k] for k in z.files}
        d["attrs"] = json.loads(str(d["attrs"]))
        return d

    @property
    def attrs(self):
        return self._load()["attrs"]

    @property
    def step(self):
        return self._load()["step"]

    @property
    def time(self):
        return self._load()["time"]

    @property
    def positions(self):
        return self._load()["positions"]

    @property
    def forces(self):
        return self._load().get("forces")

    def __len__(self):
        return len(self.step)

    def __iter__(self):
        d = self._load()
        F = d.get("forces")
        for i in range(len(d["step"])):
            yield int(d["step"][i]), float(d["time"][i]), d["positions"][i], (F[i] if F is not None else None)


class Run:
    """A run directory: the manifest plus its trajectories."""

    def __init__(self, directory):
        self.directory = directory
        with open(os.path.join(directory, "manifest.json")) as fh:
            self.manifest = json.load(fh)
        self.files = [os.path.join(directory, f) for f in self.manifest["files"]]

    def __len__(self):
        return len(self.files)

    def __iter__(self):
        for p in self.files:
            yield Trajectory(p)

    def __getitem__(self, i):
        return Trajectory(self.files[i])


def read_trajectory(path):
    return Trajectory(path)


def read_run(directory):
    return Run(directory)


def map_property(run, fn, *, use_forces=False):
    """fn(R) (or fn(R, F)) at every snapshot -> (times, values[n_traj, n_snap])."""
    times, rows = None, []
    for traj in run:
        vals, ts = [], []
        for _s, t, R, F in traj:
            vals.append(fn(R, F) if use_forces else fn(R))
            ts.append(t)
        rows.append(vals)
        if times is None:
            times = np.asarray(ts)
    return times, np.asarray(rows, dtype=float)


def ensemble_average(run, fn, *, use_forces=False):
    """(times, mean, stderr) of fn over the ensemble at each snapshot time."""
    times, values = map_property(run, fn, use_forces=use_forces)
    n = values.shape[0]
    mean = values.mean(axis=0)
    stderr = values.std(axis=0, ddof=1) / np.sqrt(n) if n > 1 else np.full(mean.shape, np.nan)
    return times, mean, stderr


class SnapshotSink:
    """Background writer: `put(path, payload)` queues a trajectory file,
    `close()` waits for all writes and re-raises the first error."""

    def __init__(self, max_pending=64):
        self.q = queue.Queue(maxsize=max_pending)
        self.err = None
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def _run(self):
        while True:
            item = self.q.get()
            if item is None:
                return
            path, kw = item
            try:
                write_trajectory(path, **kw)
            except Exception as exc:  # surfaced by close()
                if self.err is None:
                    self.err = exc

    def put(self, path, **kw):
        self.q.put((path, kw))

    def close(self):
        self.q.put(None)
        self.t.join()
        if self.err is not None:
            raise self.err


class RunWriter:
    """Chunk-by-chunk snapshot writer for a run of n_traj trajectories with
    bead offsets `offsets` (n_traj + 1) into the concatenated positions.

    put(k, step, time, positions, forces=None, ready=None): snapshot k of the
    run; positions (and forces) are host arrays (total_beads, 3), typically
    pinned tensors filled by a non-blocking device copy, and `ready` an event
    (anything with .synchronize()) recorded after that copy. The writer thread
    waits for the event, then stores the snapshot in the spool file
    (directory/.spool_*.f64, one (n_snap, total_beads, 3) float64 array).
    `release` (if given to put) is called once the buffers may be reused.

    finish(keep, attrs, compression) waits for the queue, writes
    traj_NNNNN.<ext> for every trajectory i with keep[i] (attrs(i) its
    attributes), removes the spool and returns the file names. Errors of the
    thread are raised by finish.
    """

    def __init__(self, directory, offsets, n_snap: int, write_forces: bool = False, max_pending: int = 2):
        self.directory = directory
        os.makedirs(directory, exist_ok=True)
        self.offsets = np.asarray(offsets, dtype=np.int64)
        self.n_snap = int(n_snap)
        total = int(self.offsets[-1])
        self.paths = [os.path.join(directory, ".spool_positions.f64")]
        self.pos = np.lib.format.open_memmap(self.paths[0] + ".npy", mode="w+", dtype=np.float64,
                                             shape=(self.n_snap, total, 3))
        self.paths[0] += ".npy"
        self.frc = None
        if write_forces:
            p = os.path.join(directory, ".spool_forces.f64.npy")
            self.paths.append(p)
            self.frc = np.lib.format.open_memmap(p, mode="w+", dtype=np.float64, shape=(self.n_snap, total, 3))
        self.steps = np.zeros(self.n_snap, dtype=np.int64)
        self.times = np.zeros(self.n_snap, dtype=np.float64)
        self.filled = np.zeros(self.n_snap, dtype=bool)
        self.q = queue.Queue(maxsize=max(1, int(max_pending)))
        self.err = None
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def _run(self):
        while True:
            item = self.q.get()
            if item is None:
                return
            k, step, time_, pos, frc, ready, release = item
            try:
                if ready is not None:
                    ready.synchronize()
                self.pos[k] = np.asarray(pos)
                if self.frc is not None and frc is not None:
                    self.frc[k] = np.asarray(frc)
                self.steps[k] = step
                self.times[k] = time_
                self.filled[k] = True
            except Exception as exc:  # surfaced by finish()
                if self.err is None:
                    self.err = exc
            finally:
                if release is not None:
                    release()

    def put(self, k, step, time_, positions, forces=None, ready=None, release=None):
        if not 0 <= k < self.n_snap:
            raise IndexError(f"snapshot {k} outside the run's {self.n_snap}")
        self.q.put((int(k), int(step), float(time_), positions, forces, ready, release))

    def finish(self, keep, attrs, compression="gzip", n_used=None):
        """n_used: write only the first n_used snapshots (a run cut short)."""
        self.q.put(None)
        self.t.join()
        if self.err is not None:
            raise self.err
        m = self.n_snap if n_used is None else int(n_used)
        if not self.filled[:m].all():
            raise RuntimeError("RunWriter: snapshots missing at finish")
        files = []
        for i in range(len(self.offsets) - 1):
            if not keep[i]:
                continue
            lo, hi = self.offsets[i], self.offsets[i + 1]
            path = trajectory_path(self.directory, i)
            write_trajectory(path, self.steps[:m], self.times[:m], self.pos[:m, lo:hi, :],
                             None if self.frc is None else self.frc[:m, lo:hi, :], attrs=attrs(i),
                             compression=compression)
            files.append(os.path.basename(path))
        del self.pos, self.frc
        for p in self.paths:
            os.unlink(p)
        return files
