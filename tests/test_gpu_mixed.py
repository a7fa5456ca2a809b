"""Mixed batches (families, z and depths mixed in one walk) through the C ABI
(marked gpu). Every trajectory of a mixed walk must equal, bit for bit, the
sequential walk of the same trajectory run on its own descriptor and depth:
sorting, queues, tuning and graph replay change only who walks what."""
import numpy as np
import pytest

import cmfw
import cmfw.workloads as wl

pytestmark = pytest.mark.gpu
H = 50


def _batch(n, seed):
    descs, recs, items = wl.mixed_batch(n, seed, N_lo=200, N_hi=600)
    items["N"] = np.array([200, 320, 600])[np.arange(n) % 3]
    return descs, recs, items


def _per_group(descs, recs, items, variant):
    out = np.zeros(len(recs), dtype=cmfw.OUT_DTYPE)
    for d in np.unique(items["desc"]):
        for N in np.unique(items["N"]):
            idx = np.nonzero((items["desc"] == d) & (items["N"] == N))[0]
            if len(idx):
                out[idx] = cmfw.walk(variant, descs[d], recs[idx], int(N), H, flags=cmfw.F_SEQUENTIAL)
    return out


@pytest.mark.parametrize("variant", ["f64", "df64"])
def test_mixed_equals_sequential_walks(cuda, variant):
    descs, recs, items = _batch(3000, 5)
    ref = _per_group(descs, recs, items, variant)
    assert (ref["valid"] == 1).sum() > 100
    scan = cmfw.MixedTuning()
    scan.persistent, scan.prescan = 1, 1
    for tuning in (None, cmfw.baseline_tuning(), scan):
        got = cmfw.walk_mixed(descs, recs, items, H, variant, tuning)
        assert got.tobytes() == ref.tobytes()


def test_mixed_graph_replay_and_autotune(cuda):
    descs, recs, items = _batch(2000, 9)
    ref = _per_group(descs, recs, items, "f64")
    b = cmfw.MixedBatch(descs, recs, items, H, "f64")
    t = b.autotune(sample=512)
    for f in range(len(descs)):
        assert t.tile[f].block_size in (64, 128, 256) and t.tile[f].grab in (0, 32, 64)
    b.capture(t)
    for _ in range(2):  # replays reset the queues themselves
        b.d_out.fill_(0)
        b.replay()
        assert b.results().tobytes() == ref.tobytes()
    b.release()


def test_mixed_bad_descriptor_and_depth(cuda):
    descs, recs, items = _batch(300, 3)
    items["desc"][7] = 99
    items["N"][8] = 100  # N - 2h = 0
    out, st = cmfw.walk_mixed(descs, recs, items, H, "f64", with_status=True)
    assert st[7] == 9 and out["valid"][7] == 0
    assert st[8] == 5 and out["valid"][8] == 0
    ok = np.ones(len(recs), bool)
    ok[[7, 8]] = False
    ref = _per_group(descs, recs[ok], items[ok], "f64")
    assert out[ok].tobytes() == ref.tobytes()
