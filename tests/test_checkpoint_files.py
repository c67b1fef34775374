"""Checkpoint files of batched runs (CPU): a checkpoint round-trips its next
photon index and tallies, and resumes only the batch it was taken from (the
fingerprint covers the events' parameter records, counts, first id and tally
binning)."""
import numpy as np
import pytest

from gpu_optical_photons_b200 import params as P
from gpu_optical_photons_b200.wavefront import (batch_fingerprint, batched_events, load_checkpoint,
                                                save_checkpoint)


def test_checkpoint_round_trip(tmp_path):
    events, counts = batched_events(n_events=12, seed=3, median=500)
    tc = P.TallyConfig(100, 50.0, 10)
    fp = batch_fingerprint(events, counts, 7, tc)
    t = np.arange(12 * tc.length, dtype=np.uint64).reshape(12, tc.length) * np.uint64(2**40)
    path = str(tmp_path / "c.npz")
    save_checkpoint(path, fp, 123456789012, t)
    nxt, t2 = load_checkpoint(path, fp)
    assert nxt == 123456789012
    assert t2.dtype == np.uint64 and np.array_equal(t2, t)


def test_fingerprint_tracks_the_batch(tmp_path):
    events, counts = batched_events(n_events=12, seed=3, median=500)
    tc = P.TallyConfig(100, 50.0, 10)
    fp = batch_fingerprint(events, counts, 0, tc)
    assert fp == batch_fingerprint(list(events), counts.copy(), 0, tc)
    c2 = counts.copy()
    c2[5] += 1
    e2 = list(events)
    e2[3] = e2[3].replace(abs_length=e2[3].abs_length + 1.0)
    others = [batch_fingerprint(events, c2, 0, tc), batch_fingerprint(events, counts, 1, tc),
              batch_fingerprint(e2, counts, 0, tc),
              batch_fingerprint(events, counts, 0, P.TallyConfig(100, 40.0, 10))]
    assert len({fp, *others}) == 5
    path = str(tmp_path / "c.npz")
    save_checkpoint(path, fp, 10, np.zeros((12, tc.length), np.uint64))
    with pytest.raises(ValueError, match="another batch"):
        load_checkpoint(path, others[0])


def test_checkpoint_written_under_the_given_name(tmp_path):
    """A path without the .npz extension is written as given (the next run looks
    for exactly that file), and a second save replaces the first in place with
    no temporary file left behind."""
    events, counts = batched_events(n_events=4, seed=3, median=500)
    tc = P.TallyConfig(10, 50.0, 2)
    fp = batch_fingerprint(events, counts, 0, tc)
    path = str(tmp_path / "run.ckpt")
    save_checkpoint(path, fp, 5, np.ones((4, tc.length), np.uint64))
    save_checkpoint(path, fp, 9, np.full((4, tc.length), 3, np.uint64))
    assert sorted(p.name for p in tmp_path.iterdir()) == ["run.ckpt"]
    nxt, t = load_checkpoint(path, fp)
    assert nxt == 9 and np.array_equal(t, np.full((4, tc.length), 3, np.uint64))
