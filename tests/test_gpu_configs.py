"""The benchmark configurations as configured, and the exact-verification
path, on the GPU (marked gpu):

  * the GPU exact walk's residues equal the oracle's own exact walk modulo
    the same primes (C, on the host) bit for bit, and the two verifiers
    (cmfw.exact on the GPU residues, oracle.exact_check on the oracle's)
    give the same verdicts;
  * the exact export of the top deltas round-trips to the Fraction walk;
  * valid-direction sampling keeps only directions the oracle walks validly;
  * 3F2 z = 1/2 limit starts U{1..10} (the CPU-baseline configuration);
  * 8F7 zeta RNS at N = 1000 and 4000 with 8 and 16 primes, compat
    residues bit for bit against the oracle;
  * mixed batches at depths log-uniform in 200..5000.
"""
from fractions import Fraction

import numpy as np
import pytest

import cmfw
import cmfw.workloads as wl
import oracle
from oracle import exact as fr_exact
from oracle import exact_check as ec

pytestmark = pytest.mark.gpu


def test_exact_kernel_matches_oracle_exact_walk(cuda):
    """cmfw_exact_residues against orc_exact_residues: the benchmark batch's
    valid walks (6F5 zeta, N = 1000) and 3F2 / 8F7 walks with other pairs."""
    recs = wl.zeta_directions(6, 5, 4000, 20261203)
    desc = cmfw.make_desc(6, 5, 1.0)
    out = cmfw.walk("f64", desc, recs, 1000, 50)
    sub = recs[out["valid"] == 1][:12]
    assert len(sub) >= 6
    ps = ec.primes(24)
    g, gok = cmfw.exact_residues(desc, sub, 1000, 50, ps)
    o, ook = oracle.exact_residues(6, 5, 1, 1, 1000, 50, sub, ps)
    assert np.array_equal(gok, ook)
    assert np.array_equal(g[ook[:, None, None, :].repeat(3, 1).repeat(2, 2)],
                          o[ook[:, None, None, :].repeat(3, 1).repeat(2, 2)])
    for p, q, z in ((3, 2, 0.5), (8, 7, 0.5)):
        recs = oracle.make_inputs(p, q, 90, 0, False)[:30]
        desc = cmfw.make_desc(p, q, z)
        rank = desc.rank
        pairs = np.array([((t % rank) << 8) | (((t + 1) % rank) << 4) | ((t * 7) % rank) for t in range(30)])
        g, gok = cmfw.exact_residues(desc, recs, 120, 20, ps, pairs)
        o, ook = oracle.exact_residues(p, q, *ec.z_fraction(z), 120, 20, recs, ps, pairs)
        assert np.array_equal(gok, ook), (p, q)
        mask = ook[:, None, None, :].repeat(3, 1).repeat(2, 2)
        assert np.array_equal(g[mask], o[mask]), (p, q)


def test_verifiers_agree_on_the_benchmark_batch(cuda):
    from cmfw import exact
    recs = wl.zeta_directions(6, 5, 10000, 20261203)
    desc = cmfw.make_desc(6, 5, 1.0)
    out, src = cmfw.walk("f64", desc, recs, 1000, 50, with_limit_src=True)
    a = exact.verify(desc, recs, out, src, 1000, 50, rtol=1e-10)
    b = ec.verify(6, 5, 1.0, recs, out, src, 1000, 50, rtol=1e-10)
    assert a["verified"].sum() >= 20
    assert np.array_equal(a["verified"], b["verified"])
    both = np.isfinite(a["exact_limit"]) & np.isfinite(b["exact_limit"])
    assert np.array_equal(a["exact_limit"][both], b["exact_limit"][both])


def test_export_topk_round_trips_to_the_fraction_walk(cuda):
    from cmfw import exact
    p, q, z, N, h = 3, 2, 0.5, 60, 10
    recs = wl.limit_starts(p, q, 40, 3, lo=2, hi=9)
    desc = cmfw.make_desc(p, q, z)
    out = cmfw.walk("f64", desc, recs, N, h)
    top = exact.export_topk(desc, recs, out, N, h, k=5, K0=64)
    fin = np.isfinite(out["delta"]) & (out["valid"] == 1)
    assert len(top) == min(5, int(fin.sum())) and len(top) >= 3
    deltas = [e["delta"] for e in top]
    assert deltas == sorted(deltas, reverse=True)
    assert deltas[0] == float(np.max(out["delta"][fin]))
    for e in top:
        M, snaps = fr_exact.walk(p, q, z, e["start"], e["dir"], N, snapshots=(N - 2 * h, N - h, N))
        assert M is not None and e["exact"] is not None
        for x, depth in zip(e["exact"], (N - 2 * h, N - h, N)):
            want = snaps[depth][0][2] / snaps[depth][1][2]
            assert x["depth"] == depth
            assert Fraction(int(x["num"]), int(x["den"])) == want


def test_valid_directions_are_valid_in_the_oracle(cuda):
    a = wl.valid_directions(6, 5, 60, 11, N=300, h=50, batch=1 << 14)
    b = wl.valid_directions(6, 5, 60, 11, N=300, h=50, batch=1 << 14)
    assert a.tobytes() == b.tobytes() and len(a) == 60
    o = oracle.walk("f64", 6, 5, 1.0, 300, 50, a)
    assert (o["valid"] == 1).all()
    assert (a["dir"][:, :11] >= 0).all() and (a["dir"][:, :11] <= 3).all() and a["dir"][:, :11].any(1).all()
    # the kept directions are the stream's own draws in order: a prefix of a
    # longer request
    c = wl.valid_directions(6, 5, 90, 11, N=300, h=50, batch=1 << 14)
    assert c[:60].tobytes() == a.tobytes()


def test_cfg1_limit_starts_match_oracle(cuda):
    """3F2, z = 1/2, 10,000 starts U{1..10}, direction 1^5, N = 1000, h = 50:
    the CPU-baseline configuration, validity row for row and the limits."""
    from test_gpu_walk import _exact_pq_parity, _limit_parity
    recs = wl.limit_starts(3, 2, 10000, 20261203)
    desc = cmfw.make_desc(3, 2, 0.5)
    g, src = cmfw.walk("f64", desc, recs, 1000, 50, with_limit_src=True)
    o = oracle.walk("f64", 3, 2, 0.5, 1000, 50, recs, fused=True)
    np.testing.assert_array_equal(g["valid"], o["valid"])
    m = g["valid"] == 1
    assert 0.3 < m.mean() < 0.8
    sample = np.nonzero(m)[0][:400]
    sub = np.zeros(len(recs), bool)
    sub[sample] = True
    gs, os_ = g.copy(), o.copy()
    gs["valid"][~sub] = 0
    _limit_parity(desc, recs, gs, src, os_, 1000, 50)
    _exact_pq_parity(desc, recs, g, o, sub)


@pytest.mark.parametrize("N", [1000, 4000])
@pytest.mark.parametrize("K", [8, 16])
def test_cfg3_8f7_zeta_rns(cuda, N, K):
    """8F7 at the zeta point, directions 1^15 + U{0..2}^15, compat RNS with
    K moduli: validity equal to the oracle (under the reference's path order
    the first y+ step of a zeta start is singular unless an x step comes
    first, so most trajectories are invalid) and the valid ones' limit, p
    and q bit for bit; then 8F7 z = 1/2 walks of the reference's inputs at
    the same N and K with their residue traces."""
    recs = wl.zeta_directions(8, 7, 2000, 20261203, lo=0, hi=2, offset=1)
    desc = cmfw.make_desc(8, 7, 1.0)
    g = cmfw.walk("rns", desc, recs, N, 50, n_primes=K)
    # the oracle on the rows the GPU walks validly and on 100 others
    pick = np.concatenate([np.nonzero(g["valid"] == 1)[0][:40], np.arange(100)])
    o = oracle.walk("rns", 8, 7, 1.0, N, 50, recs[pick], n_primes=K, fused=True)
    np.testing.assert_array_equal(g["valid"][pick], o["valid"])
    assert (g["valid"] == 1).mean() < 0.1  # the first y+ step of a zeta start is singular for most
    mv = o["valid"] == 1
    for k in ("limit", "p", "q"):
        assert np.array_equal(g[k][pick][mv], o[k][mv], equal_nan=True), k
    live = oracle.make_inputs(8, 7, 30, 0, False)[:8]
    desc = cmfw.make_desc(8, 7, 0.5)
    g = cmfw.walk("rns", desc, live, N, 50, n_primes=K)
    o = oracle.walk("rns", 8, 7, 0.5, N, 50, live, n_primes=K, fused=True)
    np.testing.assert_array_equal(g["valid"], o["valid"])
    m = o["valid"] == 1
    assert m.sum() >= 2
    for k in ("limit", "p", "q"):
        assert np.array_equal(g[k][m], o[k][m], equal_nan=True), k
    t = int(np.nonzero(m)[0][0])
    res, ok = cmfw.rns_trace(desc, live[t:t + 1], N, 50, K, N)
    okr, ro, _ = oracle.rns_trace(8, 7, 0.5, N, 50, live["dir"][t], live["start"][t], K, N, desc.rank,
                                  fused=True)
    assert okr == bool(ok[0])
    np.testing.assert_array_equal(ro, res[0])


def test_cfg4_mixed_depths_to_5000(cuda):
    """Mixed batch with N log-uniform in 200..5000 (the configured range):
    every trajectory equal, bit for bit, to the sequential walk of its own
    descriptor and depth."""
    descs, recs, items = wl.mixed_batch(1500, 17)
    assert items["N"].max() > 3000
    out = np.zeros(len(recs), dtype=cmfw.OUT_DTYPE)
    for d in np.unique(items["desc"]):
        for N in np.unique(items["N"][items["desc"] == d]):
            idx = np.nonzero((items["desc"] == d) & (items["N"] == N))[0]
            out[idx] = cmfw.walk("f64", descs[d], recs[idx], int(N), 50, flags=cmfw.F_SEQUENTIAL)
    got = cmfw.walk_mixed(descs, recs, items, 50, "f64")
    assert got.tobytes() == out.tobytes()
    assert (out["valid"] == 1).sum() > 20
