"""The oracle's exact path (CPU): the C exact walk modulo primes against the
Fraction walk, rational reconstruction, and the limit sources of the
oracle's restatement of the reference's reduction."""
from fractions import Fraction

import numpy as np
import pytest

import oracle
from oracle import exact as fr
from oracle import exact_check as ec

CASES = [
    (3, 2, 0.5, [3, 5, 7, 4, 6], [1, 1, 1, 1, 1]),
    (3, 2, 0.5, [5, 5, 5, 6, 6], [0, 1, 1, 1, 0]),
    (3, 2, 0.5, [2, 9, 4, 7, 3], [1, 0, 1, 0, 0]),
    (4, 3, 0.5, [2, 3, 4, 5, 3, 4, 6], [1, 0, -1, 0, 1, 0, 0]),
    (6, 5, 1.0, [1] * 6 + [2] * 5, [0, 0, 2, 1, 1, 2, 0, 0, 0, 0, 0]),
    (5, 4, 0.5, [4, 7, 2, 9, 5, 3, 8, 6, 4], [1, 0, 0, 0, 2, 0, -1, 0, 0]),
    (4, 3, 1.0, [3, 4, 2, 5, 6, 3, 4], [1, 2, 0, 1, 0, 1, -1]),
    (8, 7, 0.5, [2, 3, 4, 5, 6, 7, 8, 9, 3, 4, 5, 6, 7, 8, 9], [1] * 15),
]


def _record(p, q, start, d):
    rec = np.zeros(1, dtype=oracle.IN_DTYPE)
    rec["start"][0, :p + q] = start
    rec["dir"][0, :p + q] = d
    return rec


@pytest.mark.parametrize("p,q,z,start,d", CASES)
def test_exact_residues_match_fraction_walk(p, q, z, start, d):
    N, h = 14, 4
    rec = _record(p, q, start, d)
    ps = ec.primes(24)
    res, ok = oracle.exact_residues(p, q, *ec.z_fraction(z), N, h, rec, ps)
    M, snaps = fr.walk(p, q, z, start, d, N, snapshots=(N - 2 * h, N - h, N))
    if M is None:
        # a divisor vanished exactly: every prime sees it
        assert not ok.any()
        return
    dim = len(M)
    for s, step in enumerate((N - 2 * h, N - h, N)):
        for e, row in enumerate((0, 1)):
            val = snaps[step][row][dim - 1]
            for k, pk in enumerate(ps):
                if ok[0, k]:
                    assert int(res[0, s, e, k]) == fr.residue(val, int(pk)), (s, e, k)
    assert ok.mean() > 0.9


def test_exact_ratios_reconstruct_fraction_walk():
    for p, q, z, start, d in CASES:
        N, h = 40, 10
        rec = _record(p, q, start, d)
        M, snaps = fr.walk(p, q, z, start, d, N, snapshots=(N - 2 * h, N - h, N))
        rs = ec.exact_ratios(p, q, z, rec, N, h, K0=16)[0]
        if M is None:
            assert rs is None
            continue
        dim = len(M)
        want = [snaps[s][0][dim - 1] / snaps[s][1][dim - 1] if snaps[s][1][dim - 1] != 0 else "inf"
                for s in (N - 2 * h, N - h, N)]
        assert rs == want, (p, q, start, d)


def test_pairs_select_entries():
    p, q, z, start, d = CASES[0]
    N, h = 12, 3
    rec = _record(p, q, start, d)
    ps = ec.primes(8)
    M, snaps = fr.walk(p, q, z, start, d, N, snapshots=(N - 2 * h, N - h, N))
    assert M is not None
    i, j, c = 2, 0, 1
    res, ok = oracle.exact_residues(p, q, *ec.z_fraction(z), N, h, rec, ps,
                                    pairs=np.array([(i << 8) | (j << 4) | c]))
    for s, step in enumerate((N - 2 * h, N - h, N)):
        for k, pk in enumerate(ps):
            assert int(res[0, s, 0, k]) == fr.residue(snaps[step][i][c], int(pk))
            assert int(res[0, s, 1, k]) == fr.residue(snaps[step][j][c], int(pk))


def test_reconstruction_and_held_out_check():
    ps = ec.primes(40)
    x = Fraction(-123456789123456789, 987654321987)
    num = np.array([x.numerator % int(m) for m in ps], dtype=np.uint32)
    den = np.array([x.denominator % int(m) for m in ps], dtype=np.uint32)
    ok = np.ones(len(ps), dtype=bool)
    assert ec.ratio(num, den, ok, ps) == x
    # too few primes for this size: undetermined, never a wrong value
    assert ec.ratio(num[:7], den[:7], ok[:7], ps[:7]) is None
    assert ec.ratio(num, np.zeros_like(den), ok, ps) == "inf"
    bad = num.copy()
    bad[-1] ^= 1  # a held-out prime disagrees
    assert ec.ratio(bad, den, ok, ps) is None


def test_primes_are_the_largest_below_2_31():
    ps = ec.primes(6).tolist()
    assert ps == [2147483647, 2147483629, 2147483587, 2147483579, 2147483563, 2147483549]


def test_limit_sources_name_the_estimator():
    """walk_f64_src: the limit equals the Aitken or raw estimate of the
    ratio its source names, recomputed from the oracle's snapshots."""
    recs = oracle.make_inputs(4, 3, 60, 0, False)[:20]
    out, src = oracle.walk_f64_src(4, 3, 0.5, 200, 20, recs)
    plain = oracle.walk("f64", 4, 3, 0.5, 200, 20, recs)
    for k in ("limit", "p", "q", "delta", "valid"):
        assert np.array_equal(out[k], plain[k], equal_nan=True)
    assert ((src >= 0) <= (out["valid"] == 1)).all()
    checked = 0
    for t in np.nonzero(src >= 0)[0]:
        ok, m, _ = oracle.f64_snapshots(4, 3, 0.5, 200, 20, recs["dir"][t][:7], recs["start"][t][:7])
        i, j, c, aitken = (src[t] >> 8) & 15, (src[t] >> 4) & 15, src[t] & 15, (src[t] >> 12) & 1
        r1, r2, r3 = (m[s][i][c] / m[s][j][c] for s in range(3))
        want = r3 - (r2 - r3) ** 2 / (r1 - 2.0 * r2 + r3) if aitken else r3
        assert out["limit"][t] == want, (t, hex(src[t]))
        checked += 1
    assert checked >= 5


def test_exact_estimator_of_converged_ratios():
    q = Fraction(1, 4)
    assert ec.estimator([q, q, q], 1) == q
    assert ec.estimator([Fraction(1), Fraction(2), Fraction(3)], 1) is None
    assert ec.estimator([Fraction(1), Fraction(1, 2), Fraction(1, 3)], 0) == Fraction(1, 3)
    assert ec.estimator([Fraction(1), "inf", Fraction(1)], 0) is None
