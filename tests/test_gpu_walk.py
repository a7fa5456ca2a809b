"""GPU walks against the oracle, through the C ABI (marked gpu).

Parity bars:
  * validity flags: identical to the oracle;
  * f64 limit / p / q / log_scale: within 1e-9 relative on at least 90% of the
    valid rows and a median below 1e-12 -- the remainder are walks whose
    result is rounding noise in every build (the reference's own published
    rows show the same split, see test_oracle.py);
  * compat RNS: residues, limits, p and q bit for bit;
  * exact walk: residues equal to the Fraction walk's entries mod p;
  * df64 (accurate float-float): limits within 1e-10 of the exact value on
    convergent walks; df64 compat: within the reference's own ~1e-9 accuracy.
"""
import json
import os

import numpy as np
import pytest

import cmfw
import oracle
from oracle import exact as fr_exact

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
FAMILIES = [(3, 2), (4, 3), (5, 4), (6, 5), (8, 7)]


def _close_fraction(a, b, rtol, key, frac=0.9):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    assert (np.isfinite(a) == np.isfinite(b)).mean() >= 0.9, key
    fin = np.isfinite(a) & np.isfinite(b)
    if not fin.any():
        return
    err = np.abs(a[fin] - b[fin]) / np.maximum(np.abs(b[fin]), 1.0 if key == "log_scale" else 1e-300)
    assert (err <= rtol).mean() >= frac, (key, float(np.max(err)))
    assert np.median(err) <= 1e-11, (key, float(np.median(err)))


def _limit_parity(desc, recs, g, src, o, N, h, rtol=1e-9):
    """`limit` is the first Aitken candidate over all entry ratios, chosen by
    thresholds that sit at the rounding-noise level on converged walks, so
    two correct walks can pick different candidates, and on ill-conditioned
    walks every floating-point result carries rounding noise. Each valid row
    must agree with the oracle within rtol, or else -- arbitrated by the
    exact rational walk, against the exact value L of the GPU's own
    estimator -- be within rtol of L whenever the oracle's value is; rows
    whose estimator has no exact value (a ratio of exactly-zero entries) or
    where the oracle itself misses L are rounding noise in every build, and
    over the disagreeing rows the GPU must hit L at least as often."""
    from cmfw import exact
    m = np.nonzero(g["valid"] == 1)[0]
    gl, ol = g["limit"][m], o["limit"][m]
    both_nan = np.isnan(gl) & np.isnan(ol)
    close = both_nan | (np.abs(gl - ol) <= rtol * np.abs(ol))
    far = m[~close]
    if len(far) == 0:
        return 0
    v = exact.verify(desc, recs[far], g[far], src[far], N, h, rtol=rtol, K0=256)
    L = v["exact_limit"]
    with np.errstate(invalid="ignore", over="ignore"):
        g_ok = np.abs(g["limit"][far] - L) <= rtol * np.abs(L)
        o_ok = np.abs(o["limit"][far] - L) <= rtol * np.abs(L)
    undefined = np.isnan(L) | np.isinf(L)
    # an estimator whose rounding floor (the change of the estimate when the
    # exact ratios move by 4 ulps) is not far below rtol decides by rounding
    # which build lands within rtol
    noisy = ~(v["floor"] <= rtol / 100)
    with np.errstate(invalid="ignore", over="ignore"):
        g_err = np.abs(g["limit"][far] - L) / np.abs(L)
        o_err = np.abs(o["limit"][far] - L) / np.abs(L)
    # a row fails only where the reference's own value is exact to rtol, the
    # GPU's is not, and the GPU's error is more than ten times the
    # reference's (two walks whose errors both sit near rtol land on either
    # side of it by chance); elsewhere both are rounding noise of an
    # ill-conditioned walk (or the estimator has no exact value)
    worse = ~(g_err <= 10.0 * o_err)
    bad = far[~(g_ok | undefined | noisy | ~o_ok | ~worse)]
    assert len(bad) == 0, [(int(t), float(g["limit"][t]), float(o["limit"][t])) for t in bad[:5]]
    assert g_ok.sum() >= o_ok.sum() - 1 - len(far) // 100
    return len(far)


def _tail_parity(g, o, same_tol, tol, min_rows=0, lim_tol=1e-9):
    """precision and delta (cmf_pfq.cuh:476-552) against the oracle, on the
    valid rows whose limit the two agree on within lim_tol (the same
    estimator). Both fields take logs of differences of nearly converged
    ratios, so:
      * which rows are NaN must agree exactly (NaN comes from the structure
        of the walk: a vanishing q, log q <= 0, no finite limit);
      * rows converged to the rounding level (precision 12 or more, or
        infinite -- the ratios at N and N-h equal to the last bit -- on
        either side) carry rounding noise in both fields and are compared
        no further;
      * on the other rows infinities must agree, and the values are
        compared where well conditioned -- the ratios at N and N-h differ by
        more than 1e-6 relative, so a relative error e of the walk moves
        precision by about e * 1e6 / ln 10 digits -- and where the GPU's p/q
        agree with the oracle's within same_tol: there, within tol
        (precision, digits) and tol * max(1, |delta|) (delta) on at least 95%
        of the rows.
    Returns the number of value-compared rows."""
    m = (g["valid"] == 1) & (o["valid"] == 1)
    with np.errstate(invalid="ignore"):
        lim_same = (np.isnan(g["limit"]) & np.isnan(o["limit"])) | \
            (np.abs(g["limit"] - o["limit"]) <= lim_tol * np.abs(o["limit"]))
    m &= lim_same
    for k in ("precision", "delta"):
        assert np.array_equal(np.isnan(g[k][m]), np.isnan(o[k][m])), k
    with np.errstate(invalid="ignore"):
        converged = (np.nan_to_num(g["precision"], nan=0.0) >= 12.0) | (np.nan_to_num(o["precision"], nan=0.0) >= 12.0)
    live = m & ~converged
    for k in ("precision", "delta"):
        assert np.array_equal(np.isinf(g[k][live]), np.isinf(o[k][live])), k
    with np.errstate(invalid="ignore", divide="ignore"):
        rel_pq = np.abs(g["p"] / g["q"] - o["p"] / o["q"]) / np.abs(o["p"] / o["q"])
        scale = np.log10(np.maximum(np.abs(o["limit"]), 1e-300))
        cond = live & np.isfinite(o["precision"]) & (o["precision"] < 6.0 - scale) & (rel_pq <= same_tol)
    cond &= np.isfinite(o["delta"])
    n = int(cond.sum())
    assert n >= min_rows, n
    if n:
        dp = np.abs(g["precision"][cond] - o["precision"][cond])
        dd = np.abs(g["delta"][cond] - o["delta"][cond]) / np.maximum(1.0, np.abs(o["delta"][cond]))
        assert (dp <= tol).mean() >= 0.95, ("precision", float(dp.max()))
        assert (dd <= tol).mean() >= 0.95, ("delta", float(dd.max()))
    return n


@pytest.mark.parametrize("p,q", FAMILIES)
@pytest.mark.parametrize("z,mode", [(0.5, 0), (1.0, 0), (0.5, 1)])
@pytest.mark.parametrize("flags", [0, cmfw.F_SEQUENTIAL])
def test_f64_matches_oracle(cuda, p, q, z, mode, flags):
    zeta = z == 1.0
    recs = oracle.make_inputs(p, q, 600, mode, zeta)[:300]
    desc = cmfw.make_desc(p, q, z)
    g, st, src = cmfw.walk("f64", desc, recs, 1000, 50, flags=flags, with_status=True, with_limit_src=True)
    o = oracle.walk("f64", p, q, z, 1000, 50, recs, fused=True)
    np.testing.assert_array_equal(g["valid"], o["valid"])
    assert ((st == 0) == (g["valid"] == 1)).all()
    m = g["valid"] == 1
    if not m.any():
        return
    _limit_parity(desc, recs, g, src, o, 1000, 50)
    for k in ("p", "q", "log_scale"):
        _close_fraction(g[k][m], o[k][m], 1e-9, k)
    assert (g["n_limits"][m] == o["n_limits"][m]).mean() >= 0.8
    _tail_parity(g, o, 1e-11, 1e-4)


def test_f64_cfg2_batch_matches_oracle(cuda):
    """The benchmark's own batch (6F5 zeta, 10,000 directions U{0..3}^11,
    seed 20261203, N = 1000, h = 50): validity identical row for row, limit /
    p / q / log_scale within the oracle bars, precision and delta by their
    NaN pattern and where conditioned."""
    import cmfw.workloads as wl
    recs = wl.zeta_directions(6, 5, 10000, 20261203)
    desc = cmfw.make_desc(6, 5, 1.0)
    g, src = cmfw.walk("f64", desc, recs, 1000, 50, with_limit_src=True)
    o = oracle.walk("f64", 6, 5, 1.0, 1000, 50, recs, fused=True)
    np.testing.assert_array_equal(g["valid"], o["valid"])
    m = g["valid"] == 1
    assert 30 <= m.sum() <= 100
    _limit_parity(desc, recs, g, src, o, 1000, 50)
    _exact_pq_parity(desc, recs, g, o, m)
    _tail_parity(g, o, 1e-11, 1e-4)


def _exact_pq_parity(desc, recs, g, o, m, n_max=300):
    """p / q at depth N against the exact ratio on (up to n_max of) the
    rows m: where many walks are ill-conditioned (the exact q many orders
    below the matrix norm) the oracle's sequential f64 walk is no reference
    for p and q, so both are compared with the exact value -- the GPU is
    within 1e-12 and 1e-10 on at least as many rows as the oracle -- and
    log_scale is compared where the two agree on p / q."""
    from cmfw import exact
    with np.errstate(invalid="ignore", divide="ignore"):
        same = np.abs(g["p"] / g["q"] - o["p"] / o["q"]) <= 1e-9 * np.abs(o["p"] / o["q"])
    both = m & same
    if both.any():
        _close_fraction(g["log_scale"][both], o["log_scale"][both], 1e-9, "log_scale")
    idx = np.nonzero(m & (g["q"] != 0) & (o["q"] != 0))[0][:n_max]
    ratios, _ = exact.exact_ratios(desc, recs[idx], 1000, 50, K0=1024)
    eg, eo = [], []
    for t, rs in zip(idx, ratios):
        if rs is None or rs[2] == "inf" or rs[2] == 0:
            continue
        ex = float(rs[2])
        eg.append(abs(g["p"][t] / g["q"][t] - ex) / abs(ex))
        eo.append(abs(o["p"][t] / o["q"][t] - ex) / abs(ex))
    eg, eo = np.array(eg), np.array(eo)
    assert len(eg) >= 20
    for bar in (1e-12, 1e-10):
        assert (eg <= bar).sum() >= (eo <= bar).sum(), (bar, eg.tolist(), eo.tolist())


def test_df64_tail_matches_oracle(cuda):
    """df64 (float-float runs): precision and delta against the oracle's f64
    walk, NaN pattern exactly, values where conditioned (a float-float walk
    is good to about 1e-9 relative, so the bar is 1e-3)."""
    p, q = 4, 3
    recs = oracle.make_inputs(p, q, 600, 0, False)[:300]
    desc = cmfw.make_desc(p, q, 0.5)
    g = cmfw.walk("df64", desc, recs, 1000, 50)
    o = oracle.walk("f64", p, q, 0.5, 1000, 50, recs, fused=True)
    np.testing.assert_array_equal(g["valid"], o["valid"])
    _tail_parity(g, o, 1e-8, 1e-3, lim_tol=1e-6)


@pytest.mark.parametrize("p,q", [(6, 5), (8, 7), (3, 2)])
@pytest.mark.parametrize("flags", [0, cmfw.F_SEQUENTIAL])
def test_f64_accuracy_vs_exact(cuda, p, q, flags):
    """Raw ratio p/q at depth N against the exact ratio over the valid rows:
    the GPU (chunked walk with double-double runs, or the sequential walk)
    keeps at least as many rows within 1e-12 and within 1e-10 as the
    reference's own kernel body (host build). Row by row both are rounding
    noise on ill-conditioned walks, so the comparison is over the rows."""
    from cmfw import exact
    recs = oracle.make_inputs(p, q, 600, 0, False)[:300]
    desc = cmfw.make_desc(p, q, 0.5)
    g = cmfw.walk("f64", desc, recs, 1000, 50, flags=flags)
    o = oracle.walk("f64", p, q, 0.5, 1000, 50, recs)
    m = np.nonzero((g["valid"] == 1) & (o["valid"] == 1) & (g["q"] != 0) & (o["q"] != 0))[0][:150]
    ratios, _ = exact.exact_ratios(desc, recs[m], 1000, 50, K0=1024)
    eg, eo = [], []
    for t, rs in zip(m, ratios):
        if rs is None or rs[2] == "inf" or rs[2] == 0:
            continue
        ex = float(rs[2])
        eg.append(abs(g["p"][t] / g["q"][t] - ex) / abs(ex))
        eo.append(abs(o["p"][t] / o["q"][t] - ex) / abs(ex))
    eg, eo = np.array(eg), np.array(eo)
    assert len(eg) >= 20
    slack = 1 if flags == 0 else max(2, len(eg) // 50)
    for bar in (1e-12, 1e-10):
        assert (eg <= bar).sum() >= (eo <= bar).sum() - slack, (bar, int((eg <= bar).sum()), int((eo <= bar).sum()))


def test_f64_zeta_limit_tight(cuda):
    """Zeta-start limit walks are well conditioned: every row within 1e-11."""
    for p, q in FAMILIES:
        recs = oracle.make_inputs(p, q, 50, 0, True)
        desc = cmfw.make_desc(p, q, 1.0)
        g = cmfw.walk("f64", desc, recs, 1000, 50)
        o = oracle.walk("f64", p, q, 1.0, 1000, 50, recs, fused=True)
        for k in ("limit", "p", "q"):
            np.testing.assert_allclose(g[k], o[k], rtol=1e-11, atol=0)
        np.testing.assert_allclose(g["log_scale"], o["log_scale"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("p,q,z,zeta", [(3, 2, 0.5, False), (4, 3, 1.0, True), (5, 4, 0.5, False),
                                        (6, 5, 1.0, True), (8, 7, 0.5, False)])
@pytest.mark.parametrize("fused", [True, False])
def test_rns_compat_bitwise(cuda, p, q, z, zeta, fused):
    recs = oracle.make_inputs(p, q, 200, 0, zeta)[:48]
    desc = cmfw.make_desc(p, q, z)
    flags = 0 if fused else cmfw.F_UNFUSED_COLUMN
    for K in (8, 13, 64):
        g = cmfw.walk("rns", desc, recs, 300, 50, n_primes=K, flags=flags)
        o = oracle.walk("rns", p, q, z, 300, 50, recs, n_primes=K, fused=fused)
        np.testing.assert_array_equal(g["valid"], o["valid"])
        m = o["valid"] == 1
        for k in ("limit", "p", "q"):
            assert np.array_equal(g[k][m], o[k][m], equal_nan=True), (K, k)
        np.testing.assert_array_equal(g["n_limits"][m], o["n_limits"][m])
        # log-derived fields: the device and host log/log10 may differ by an ulp
        for k in ("precision", "delta", "log_scale"):
            np.testing.assert_allclose(g[k][m], o[k][m], rtol=1e-12, atol=0, equal_nan=True, err_msg=k)


def test_rns_residue_traces_match_reference_golden(cuda):
    with open(os.path.join(GOLD, "reference_host_runs.json")) as f:
        cases = [c for c in json.load(f) if c["kind"] == "rns_trace"]
    assert cases
    for c in cases:
        rec = np.zeros(1, dtype=cmfw.IN_DTYPE)
        rec["dir"][0, :len(c["dir"])] = c["dir"]
        rec["start"][0, :len(c["start"])] = c["start"]
        desc = cmfw.make_desc(c["p"], c["q"], c["z"])
        flags = 0 if c["fused"] else cmfw.F_UNFUSED_COLUMN
        res, ok = cmfw.rns_trace(desc, rec, c["N"], c["h"], c["n_primes"], c["steps"], flags)
        assert bool(ok[0]) == c["ok"]
        assert res[0].reshape(-1).tolist() == c["residues"], (c["p"], c["q"], c["n_primes"], c["fused"])


def test_rns_trace_matches_oracle_many(cuda):
    rng = np.random.default_rng(5)
    desc = cmfw.make_desc(3, 2, 0.5)
    recs = np.zeros(64, dtype=cmfw.IN_DTYPE)
    recs["start"][:, :5] = rng.integers(2, 12, (64, 5))
    recs["dir"][:, :5] = rng.integers(0, 2, (64, 5))
    recs["dir"][:, 0] = 1
    res, ok = cmfw.rns_trace(desc, recs, 300, 50, 24, 130)
    for i in range(64):
        okr, ro, _ = oracle.rns_trace(3, 2, 0.5, 300, 50, recs["dir"][i], recs["start"][i], 24, 130, 3,
                                      fused=True)
        assert okr == bool(ok[i])
        if okr:
            np.testing.assert_array_equal(ro, res[i])


@pytest.mark.parametrize("p,q,z,start,d", [
    (3, 2, 0.5, [3, 5, 7, 4, 6], [1, 1, 1, 1, 1]),
    (3, 2, 0.5, [5, 5, 5, 6, 6], [0, 1, 1, 1, 0]),
    (4, 3, 0.5, [2, 3, 4, 5, 3, 4, 6], [1, 0, -1, 0, 1, 0, 0]),
    (6, 5, 1.0, [1] * 6 + [2] * 5, [0, 0, 2, 1, 1, 2, 0, 0, 0, 0, 0]),
    (5, 4, 0.5, [4, 7, 2, 9, 5, 3, 8, 6, 4], [1, 0, 0, 0, 2, 0, -1, 0, 0]),
])
def test_exact_residues_match_fraction_walk(cuda, p, q, z, start, d):
    from cmfw import exact
    N, h = 16, 4
    rec = np.zeros(1, dtype=cmfw.IN_DTYPE)
    rec["start"][0, :p + q] = start
    rec["dir"][0, :p + q] = d
    desc = cmfw.make_desc(p, q, z)
    primes = exact.primes_below_2_31(40)
    res, ok = cmfw.exact_residues(desc, rec, N, h, primes.astype(np.uint32))
    M, snaps = fr_exact.walk(p, q, z, start, d, N, snapshots=(N - 2 * h, N - h, N))
    if M is None:
        assert not ok[0].any()
        return
    dim = desc.rank
    for s, step in enumerate((N - 2 * h, N - h, N)):
        for e, row in enumerate((0, 1)):
            val = snaps[step][row][dim - 1]
            for k, pk in enumerate(primes):
                if ok[0, k]:
                    assert int(res[0, s, e, k]) == fr_exact.residue(val, int(pk)), (s, e, k)
    assert ok[0].mean() > 0.9


def test_exact_ratios_reconstruct_fraction_walk(cuda):
    from cmfw import exact
    p, q, z = 3, 2, 0.5
    rec = np.zeros(2, dtype=cmfw.IN_DTYPE)
    rec["start"][0, :5] = [3, 5, 7, 4, 6]
    rec["dir"][0, :5] = [1, 1, 1, 1, 1]
    rec["start"][1, :5] = [2, 9, 4, 7, 3]
    rec["dir"][1, :5] = [1, 0, 1, 0, 0]
    N, h = 60, 10
    desc = cmfw.make_desc(p, q, z)
    ratios, K = exact.exact_ratios(desc, rec, N, h, K0=256)
    for i in range(2):
        M, snaps = fr_exact.walk(p, q, z, rec["start"][i], rec["dir"][i], N, snapshots=(40, 50, 60))
        want = [snaps[s][0][2] / snaps[s][1][2] for s in (40, 50, 60)]
        assert ratios[i] == want


def test_verified_limits_cfg2_subset(cuda):
    """6F5 zeta: the f64 limits that verify do so within 1e-10; a known
    trajectory (dir 0,0,2,1,1,2 on x) has p/q = 1/4 exactly at every depth."""
    import cmfw.workloads as wl
    from cmfw import exact
    recs = wl.zeta_directions(6, 5, 2000, 20261203)
    extra = np.zeros(1, dtype=cmfw.IN_DTYPE)
    extra["start"][0, :11] = wl.zeta_start(6, 5)
    extra["dir"][0, :11] = [0, 0, 2, 1, 1, 2, 0, 0, 0, 0, 0]
    recs = np.concatenate([extra, recs])
    desc = cmfw.make_desc(6, 5, 1.0)
    out, src = cmfw.walk("f64", desc, recs, 1000, 50, with_limit_src=True)
    assert out["valid"][0] == 1
    v = exact.verify(desc, recs, out, src, 1000, 50)
    assert v["verified"][0] and v["exact_limit"][0] == 0.25
    valid = out["valid"] == 1
    assert v["verified"].sum() >= 1
    assert (v["rel_err"][v["verified"]] <= 1e-10).all()
    assert not v["verified"][~valid].any()


def test_df64_accurate_against_exact(cuda):
    """Convergent 3F2 walks against the exact ratio p/q at depth N: the f64
    walk keeps at least as many rows within 1e-11 as the reference's own f64
    kernel body, and the accurate float-float walk (48-bit significands) at
    least as many within 1e-9 as the reference's df64 arithmetic, with a
    median error below 1e-9."""
    from cmfw import exact
    import cmfw.workloads as wl
    recs = wl.limit_starts(3, 2, 64, 11, lo=2, hi=9)
    desc = cmfw.make_desc(3, 2, 0.5)
    g64 = cmfw.walk("f64", desc, recs, 300, 30)
    gff = cmfw.walk("df64", desc, recs, 300, 30)
    o64 = oracle.walk("f64", 3, 2, 0.5, 300, 30, recs, fused=True)
    off = oracle.walk("df64", 3, 2, 0.5, 300, 30, recs, fused=True)
    np.testing.assert_array_equal(g64["valid"], gff["valid"])
    m = np.nonzero((g64["valid"] == 1) & (off["valid"] == 1))[0]
    assert len(m) >= 5
    ratios, _ = exact.exact_ratios(desc, recs[m], 300, 30, K0=256)
    err = {k: [] for k in ("g64", "gff", "o64", "off")}
    for t, rs in zip(m, ratios):
        if rs is None or rs[2] == "inf" or rs[2] == 0:
            continue
        ex = float(rs[2])
        for k, r in (("g64", g64), ("gff", gff), ("o64", o64), ("off", off)):
            err[k].append(abs(r["p"][t] / r["q"][t] - ex) / abs(ex))
    e = {k: np.array(v) for k, v in err.items()}
    assert len(e["g64"]) >= 5
    assert (e["g64"] <= 1e-11).sum() >= (e["o64"] <= 1e-11).sum(), (e["g64"].tolist(), e["o64"].tolist())
    assert (e["gff"] <= 1e-9).sum() >= (e["off"] <= 1e-9).sum(), (e["gff"].tolist(), e["off"].tolist())
    assert np.median(e["gff"]) <= 1e-9


@pytest.mark.parametrize("p,q", FAMILIES)
@pytest.mark.parametrize("z,mode,zeta", [(1.0, 0, True), (0.5, 0, False), (0.5, 1, False)])
def test_df64_compat_matches_oracle(cuda, p, q, z, mode, zeta):
    """The reference's own df64 arithmetic (float reciprocals,
    cmf_walk_df64.cu:35-349) on the GPU against the oracle's restatement of
    it: validity identical; p and q within 1e-7 on the valid rows where the
    walk is conditioned well enough for a ~1e-9 arithmetic (the oracle's own
    f64 walk agrees with its df64 walk to 1e-6) -- elsewhere both are
    rounding noise of a 48-bit walk; the limit within 1e-7 on at least 60%
    of those rows: compute_limits picks the first candidate whose second
    difference clears a threshold at the rounding level (cmf_pfq.cuh:385-460),
    and a ~1e-9 arithmetic puts converged walks' differences right at it, so
    two builds pick different candidates on a third of these rows even
    though their walks (p, q) agree."""
    recs = oracle.make_inputs(p, q, 300, mode, zeta)[:100]
    desc = cmfw.make_desc(p, q, z)
    g = cmfw.walk("df64", desc, recs, 1000, 50, flags=cmfw.F_DF64_COMPAT)
    o = oracle.walk("df64", p, q, z, 1000, 50, recs, fused=True)
    o64 = oracle.walk("f64", p, q, z, 1000, 50, recs, fused=True)
    np.testing.assert_array_equal(g["valid"], o["valid"])
    m = (o["valid"] == 1) & np.isfinite(o["limit"]) & np.isfinite(o64["limit"])
    with np.errstate(invalid="ignore"):
        m &= np.abs(o["limit"] - o64["limit"]) <= 1e-6 * np.abs(o64["limit"])
        m &= np.abs(o["q"] - o64["q"]) <= 1e-6 * np.abs(o64["q"])
    if not m.any():
        return
    np.testing.assert_allclose(g["q"][m], o["q"][m], rtol=1e-7)
    np.testing.assert_allclose(g["p"][m], o["p"][m], rtol=1e-7, atol=1e-12)
    with np.errstate(invalid="ignore"):
        same = np.abs(g["limit"][m] - o["limit"][m]) <= 1e-7 * np.abs(o["limit"][m])
    assert same.mean() >= 0.6, (int(same.sum()), int(m.sum()))


@pytest.mark.parametrize("variant,rtol", [("f64", 1e-11), ("df64", 1e-9)])
def test_chunk_parts_agree(cuda, variant, rtol):
    """The chunked walk spreads each survivor over as many CTAs as the batch
    leaves room for (1 to 16 parts, combined by the last part to finish,
    more for costlier walks) and cuts runs inside lattice steps; every batch
    size gives a different association of the same product. Zeta-start
    limit walks are well conditioned, so every batch size -- every part
    count -- must give the oracle's limit, p and q to rtol."""
    for p, q in [(6, 5), (3, 2), (8, 7)]:
        recs = oracle.make_inputs(p, q, 200, 0, True)
        desc = cmfw.make_desc(p, q, 1.0)
        o = oracle.walk("f64", p, q, 1.0, 1000, 50, recs, fused=True)
        assert (o["valid"] == 1).all()
        for n in (1, 3, 20, 40, 60, 200):  # 16, 16, 7, 3, 2 and 1 parts on 148 SMs
            g = cmfw.walk(variant, desc, recs[:n], 1000, 50)
            np.testing.assert_array_equal(g["valid"], o["valid"][:n])
            for k in ("limit", "p", "q"):
                np.testing.assert_allclose(g[k], o[k][:n], rtol=rtol, atol=0, err_msg=f"{p}F{q} n={n} {k}")


def test_zero_direction_walks_nowhere(cuda):
    """A zero direction has no axis steps: every run of the chunked walk is
    empty and the snapshots are the identity, as in the oracle."""
    desc = cmfw.make_desc(3, 2, 0.5)
    recs = oracle.make_inputs(3, 2, 8, 0, False)[:4].copy()
    recs["dir"][2, :] = 0
    o = oracle.walk("f64", 3, 2, 0.5, 200, 20, recs, fused=True)
    for flags in (0, cmfw.F_SEQUENTIAL):
        g = cmfw.walk("f64", desc, recs, 200, 20, flags=flags)
        np.testing.assert_array_equal(g["valid"], o["valid"])
        for k in ("limit", "p", "q", "log_scale"):
            np.testing.assert_allclose(g[k], o[k], rtol=1e-12, atol=0, equal_nan=True, err_msg=k)


def test_non_dyadic_starts_match_the_oracle(cuda):
    """Starts that are not dyadic (3.7, 1.3, ...): the filter and the runs
    form positions in closed form (start plus the moves so far), which is
    the step-by-step walk's value for dyadic starts and within an ulp of it
    otherwise, like the FMA contraction of the column; a test that lands
    within an ulp of its threshold may then decide the other way. Validity
    agrees on all but a few rows. With non-integer columns every step
    rounds, and q (an entry of the normalised matrix) is far below the
    matrix scale on some rows, where the sequential f64 walk of the oracle
    and the double-double chunked walk part by up to about 1e-3 (measured:
    20 of 221 rows beyond 1e-9); most rows agree within 1e-9."""
    rng = np.random.default_rng(5)
    n = 300
    recs = np.zeros(n, dtype=cmfw.IN_DTYPE)
    recs["start"][:, :5] = np.round(rng.uniform(1.0, 9.0, (n, 5)), 1)
    recs["dir"][:, :5] = rng.integers(-2, 3, (n, 5))
    recs["dir"][:, 0] = np.where((recs["dir"][:, :5] == 0).all(1), 1, recs["dir"][:, 0])
    desc = cmfw.make_desc(3, 2, 0.5)
    o = oracle.walk("f64", 3, 2, 0.5, 200, 20, recs, fused=True)
    g = cmfw.walk("f64", desc, recs, 200, 20)
    assert 0 < (o["valid"] == 1).sum() < n
    assert (g["valid"] == o["valid"]).mean() >= 0.98, (g["valid"] != o["valid"]).sum()
    v = (o["valid"] == 1) & (g["valid"] == 1)
    rel = np.abs(g["q"][v] - o["q"][v]) / np.abs(o["q"][v])
    assert (rel <= 1e-9).mean() >= 0.85 and rel.max() <= 1e-2, (np.sort(rel)[-5:], (rel > 1e-9).sum())


def test_failure_statuses(cuda):
    desc = cmfw.make_desc(3, 2, 0.5)
    recs = oracle.make_inputs(3, 2, 8, 0, False)[:8].copy()
    recs["dir"][1, 0] = 5000          # beyond CMFW_MAX_DIR_COMPONENT
    recs["start"][2, :5] = [1, 1, 1, 1, 1]
    recs["dir"][2, :5] = [0, 0, 0, 0, -1]   # y- step with y = 1: denominator 0
    out, st = cmfw.walk("f64", desc, recs, 100, 10, with_status=True)
    assert st[1] == 6 and out["valid"][1] == 0
    assert st[2] == 2 and out["valid"][2] == 0
    out, st = cmfw.walk("f64", desc, recs, 20, 10, with_status=True)  # N - 2h = 0
    # the direction cap is checked first, then the depths
    assert st[1] == 6 and (np.delete(st, 1) == 5).all() and (out["valid"] == 0).all()
    assert np.isnan(out["limit"]).all()


def test_empty_batch_and_caller_workspace(cuda):
    import torch
    desc = cmfw.make_desc(3, 2, 0.5)
    assert len(cmfw.walk("f64", desc, np.zeros(0, dtype=cmfw.IN_DTYPE), 100, 10)) == 0
    recs = oracle.make_inputs(3, 2, 64, 0, False)
    d_in = cmfw.to_device(recs)
    need = cmfw.lib().cmfw_walk_workspace_bytes(desc, len(recs))
    ws = torch.empty(need, dtype=torch.uint8, device="cuda")
    d_out = cmfw.out_buffer(len(recs))
    cmfw.launch_walk("f64", desc, d_in, d_out, len(recs), 200, 20, d_workspace=ws)
    torch.cuda.synchronize()
    a = cmfw.records_from_device(d_out, len(recs))
    b = cmfw.walk("f64", desc, recs, 200, 20)
    assert a.tobytes() == b.tobytes()
    small = torch.empty(need // 2, dtype=torch.uint8, device="cuda")
    with pytest.raises(cmfw.CmfwError, match="EINVAL"):
        cmfw.launch_walk("f64", desc, d_in, d_out, len(recs), 200, 20, d_workspace=small)


def test_main_kernel_events(cuda):
    """launch.ev_main_start/stop: the library records them around the walk's
    main kernel (the chunk kernel, or the sequential kernel), so their
    interval is positive and inside the whole call's; results unchanged."""
    torch = cuda
    desc = cmfw.make_desc(6, 5, 1.0)
    recs = oracle.make_inputs(6, 5, 600, 0, True)[:300]
    n = len(recs)
    d_in, d_out = cmfw.to_device(recs), cmfw.out_buffer(n)
    ref = cmfw.walk("f64", desc, recs, 300, 30)
    for flags in (0, cmfw.F_SEQUENTIAL):
        kev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        whole = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        for e in kev:
            e.record()
        whole[0].record()
        cmfw.launch_walk("f64", desc, d_in, d_out, n, 300, 30, flags=flags, main_events=kev)
        whole[1].record()
        torch.cuda.synchronize()
        k_ms, w_ms = kev[0].elapsed_time(kev[1]), whole[0].elapsed_time(whole[1])
        assert 0 < k_ms <= w_ms, (flags, k_ms, w_ms)
        out = cmfw.records_from_device(d_out, n)
        if flags == 0:
            assert out.tobytes() == ref.tobytes()


def test_host_entry_point_matches_device_entry(cuda):
    desc = cmfw.make_desc(5, 4, 0.5)
    recs = oracle.make_inputs(5, 4, 300, 0, False)[:200]
    for variant in ("f64", "df64", "rns"):
        a, kms, tms = cmfw.walk_host(variant, desc, recs, 300, 30)
        b = cmfw.walk(variant, desc, recs, 300, 30)
        assert a.tobytes() == b.tobytes()
        assert 0 < kms <= tms
