"""Host-side tools around the walk (CPU only): the sweep's result tables,
the checkpointed runner's resume logic, the seeded stream, and the
exact-verification helpers (CRT, rational reconstruction) on synthetic
residues."""
import csv
import io
import os
from fractions import Fraction

import numpy as np
import pytest

import cmfw
import oracle
from cmfw import exact, runner, sweep


def test_sweep_tables_have_the_reference_runner_columns(tmp_path):
    rows = [{"cmf": "3F2", "variant": "f64", "mode": "limit", "rank": 3, "N": 1000, "h": 50, "n_traj": 10,
             "gpu_time_ms": 1.5, "throughput_traj_per_s": 6666.7, "mem_used_mb": 12.0, "n_valid": 5,
             "n_with_limits": 5, "avg_delta": None, "wall_time_s": 0.2}]
    sweep.write_tables(rows, tmp_path)
    text = (tmp_path / "benchmark_table.csv").read_text()
    header = next(csv.reader(io.StringIO(text)))
    # benchmarks/run_benchmark.py:143-145
    assert header == ["cmf", "variant", "mode", "rank", "N", "h", "n_traj", "gpu_time_ms", "throughput_traj_s",
                      "mem_mb", "n_valid", "n_with_limits", "avg_delta", "wall_time_s"]
    assert text.splitlines()[1] == "3F2,f64,limit,3,1000,50,10,1.500,6666.7,12.00,5,5,None,0.200"
    md = (tmp_path / "benchmark_table.md").read_text()
    assert "| 3F2 | f64 | limit | 3 | 1.5 | 6667 | 12.0 | 5/10 | 5 | None |" in md


def test_checkpointed_runner_resumes(tmp_path, monkeypatch):
    calls = []

    def fake_walk(variant, desc, recs, N, h, n_primes=8, flags=0):
        calls.append(len(recs))
        out = oracle.walk("f64", desc.p, desc.q, desc.z, N, h, recs, threads=1)
        res = np.zeros(len(recs), dtype=cmfw.OUT_DTYPE)
        for k in cmfw.OUT_DTYPE.names:
            res[k] = out[k]
        return res

    monkeypatch.setattr(runner.api, "walk", fake_walk)
    desc = cmfw.make_desc(3, 2, 0.5)
    recs = cmfw.reference_inputs(3, 2, 100, 0, False)
    state = str(tmp_path / "state")

    def boom(i, n):
        if i == 2:
            raise KeyboardInterrupt

    with pytest.raises(KeyboardInterrupt):
        runner.run_checkpointed("f64", desc, recs, 200, 20, 25, state, on_chunk=boom)
    assert calls == [25, 25, 25]
    done = open(os.path.join(state, "done.bin"), "rb").read()
    assert list(done) == [1, 1, 1, 0]
    calls.clear()
    out, walked = runner.run_checkpointed("f64", desc, recs, 200, 20, 25, state)
    assert calls == [25] and walked == 1
    full = fake_walk("f64", desc, recs, 200, 20)
    assert out.tobytes() == full.tobytes()
    with pytest.raises(ValueError):
        runner.run_checkpointed("f64", desc, recs, 300, 20, 25, state)


def test_mt64_stream_pieces_join():
    whole = cmfw.mt64(7, 1000)
    assert np.array_equal(np.concatenate([cmfw.mt64(7, 300), cmfw.mt64(7, 700, offset=300)]), whole)
    assert np.array_equal(whole, oracle.mt64_stream(7, 1000))
    from cmfw.workloads import _Stream
    s = _Stream(7, chunk=64)
    assert np.array_equal(np.concatenate([s.take(100), s.take(1), s.take(899)]), whole)


def test_rational_reconstruction_from_residues():
    primes = exact.primes_below_2_31(24)
    assert all(int(p) < 2 ** 31 for p in primes) and len(set(primes.tolist())) == 24
    for num, den in [(1, 4), (-355, 113), (2 ** 200 + 7, 3 ** 90), (0, 1)]:
        fr = Fraction(num, den)
        a = np.array([fr.numerator % int(p) for p in primes], dtype=np.uint32)
        b = np.array([fr.denominator % int(p) for p in primes], dtype=np.uint32)
        ok = np.ones(24, dtype=bool)
        got = exact._ratio_from_residues(a, b, ok, primes)
        if abs(fr.numerator).bit_length() + fr.denominator.bit_length() < 20 * 31 - 2:
            assert got == fr
        else:
            assert got is None  # not determined by 20 primes: the caller adds primes
    # a vanishing denominator on every prime is an exact zero
    z = np.zeros(24, dtype=np.uint32)
    assert exact._ratio_from_residues(np.ones(24, np.uint32), z, np.ones(24, bool), primes) == "inf"


def test_exact_estimator_matches_reference_formula():
    r = [Fraction(1, 3), Fraction(1, 4), Fraction(1, 5)]
    den = r[0] - 2 * r[1] + r[2]
    assert exact.exact_estimator(r, 1) == r[2] - (r[1] - r[2]) ** 2 / den
    assert exact.exact_estimator(r, 0) == r[2]
    same = [Fraction(1, 4)] * 3
    assert exact.exact_estimator(same, 1) == Fraction(1, 4)
    assert exact.exact_estimator(None, 1) is None


def test_proposal_helpers():
    from cmfw import proposal as prop
    valid = np.array([1, 1, 1, 0, 1, 1, 1, 1], bool)
    delta = np.array([0.5, 9.0, np.nan, 99.0, 3.0, -1.0, 7.0, np.inf])
    t, w, thr = prop.top_target(valid, delta, top_q=0.2)
    # finite deltas of valid walks: 0.5, 9, 3, -1, 7; the top 20% is 9
    assert thr == np.quantile([0.5, 9.0, 3.0, -1.0, 7.0], 0.8)
    assert t.tolist() == [0, 1, 0, 0, 0, 0, 0, 0] and t.dtype == np.float32
    assert w[1] == 7.0 and (np.delete(w, 1) == 1.0).all()
    idx, d = prop.top_k(np.array([10, 11, 12, 13]), np.array([0.5, 3.0, -1.0, 3.0]), 2)
    assert idx.tolist() == [11, 13] and d.tolist() == [3.0, 3.0]
    assert prop.recall([1, 2, 3], [3, 4]) == 0.5
    assert prop.recall([], []) == 1.0


def test_top_k_ties_rank_by_index_in_sweep_and_proposal():
    # the sweep walks the survivors in ascending index order and the
    # proposal walks the ones it chose in the same order, so equal deltas
    # at the cut are taken alike by both top-k lists
    from cmfw import proposal as prop
    idx = np.array([4, 7, 9, 12, 15])
    d = np.array([2.0, 5.0, 5.0, 5.0, 1.0])
    sw_i, _ = prop.top_k(idx, d, 2)
    assert sw_i.tolist() == [7, 9]
    chosen = np.array([3, 1, 2])  # positions a selection returned, in its own order
    pr_i, _ = prop.top_k(idx[np.sort(chosen)], d[np.sort(chosen)], 2)
    assert pr_i.tolist() == sw_i.tolist()
    unsorted_i, _ = prop.top_k(idx[chosen], d[chosen], 2)
    assert unsorted_i.tolist() != sw_i.tolist()


def test_mixed_batch_generator():
    import cmfw.workloads as wl
    d1, r1, i1 = wl.mixed_batch(500, 3)
    d2, r2, i2 = wl.mixed_batch(500, 3)
    assert r1.tobytes() == r2.tobytes() and i1.tobytes() == i2.tobytes()
    assert len(d1) == 10 and i1["desc"].min() >= 0 and i1["desc"].max() <= 9
    assert i1["N"].min() >= 200 and i1["N"].max() < 5000
    for t in range(500):
        p, q = wl.MIXED_FAMILIES[i1["desc"][t] // 2]
        assert r1["dir"][t, :p + q].any() and not r1["dir"][t, p + q:].any()
        assert ((r1["start"][t, :p + q] >= 1) & (r1["start"][t, :p + q] <= 10)).all()
