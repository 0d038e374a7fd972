"""The run directory writers (bdsim_b200.storage) without a GPU: snapshots
spooled chunk by chunk by RunWriter give the files write_trajectory gives for
the whole trajectory at once, in the layout of python/bdsim/storage.py."""
import os

import numpy as np

from bdsim_b200 import storage


class _Ready:
    def __init__(self):
        self.waited = False

    def synchronize(self):
        self.waited = True


def test_run_writer_spools_chunks_into_per_trajectory_files(tmp_path):
    rng = np.random.default_rng(0)
    Ns = [5, 7, 3]
    off = np.concatenate([[0], np.cumsum(Ns)])
    n_snap = 4
    pos = rng.normal(size=(n_snap, off[-1], 3))
    frc = rng.normal(size=(n_snap, off[-1], 3))
    w = storage.RunWriter(str(tmp_path / "run"), off, n_snap, write_forces=True, max_pending=1)
    readies, released = [], []
    for k in range(n_snap):
        r = _Ready()
        readies.append(r)
        w.put(k, 10 * k, 0.5 * k, pos[k].copy(), frc[k].copy(), ready=r, release=lambda k=k: released.append(k))
    files = w.finish([True, False, True], lambda i: {"index": i})
    assert all(r.waited for r in readies) and sorted(released) == list(range(n_snap))
    assert files == [os.path.basename(storage.trajectory_path(str(tmp_path / "run"), i)) for i in (0, 2)]
    assert not any(f.startswith(".spool") for f in os.listdir(tmp_path / "run"))
    for i in (0, 2):
        t = storage.read_trajectory(storage.trajectory_path(str(tmp_path / "run"), i))
        assert list(t.step) == [0, 10, 20, 30] and np.allclose(t.time, [0.0, 0.5, 1.0, 1.5])
        assert np.array_equal(t.positions, pos[:, off[i]:off[i + 1]])
        assert np.array_equal(t.forces, frc[:, off[i]:off[i + 1]])
        assert t.attrs["index"] == i and t.attrs["has_forces"]


def test_run_writer_keeps_the_snapshots_of_a_run_cut_short(tmp_path):
    off = np.array([0, 4])
    w = storage.RunWriter(str(tmp_path), off, 5)
    for k in range(2):
        w.put(k, k, float(k), np.full((4, 3), float(k)))
    files = w.finish([True], lambda i: {}, n_used=2)
    t = storage.read_trajectory(os.path.join(str(tmp_path), files[0]))
    assert list(t.step) == [0, 1] and t.positions.shape == (2, 4, 3) and t.forces is None
