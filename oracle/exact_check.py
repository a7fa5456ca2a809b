"""Exact values of the reference's limit estimators -- TEST INFRASTRUCTURE.

The checker's own exact path, independent of the product library: the C
exact walk modulo primes (``orc_exact_residues`` in cmfw_oracle.c) gives the
residues of two entries of one column of the walk matrix at depths N-2h,
N-h and N; here each ratio M[i][c] / M[j][c] becomes an exact rational
(per prime a * b^-1, Chinese remaindering, rational reconstruction with the
bound sqrt(P/2) of Wang's method, confirmed on held-out primes), and a
floating-point limit is compared with the exact value of the estimator it
came from (the Aitken or raw estimate of the reference's reduction,
cmf_pfq.cuh:385-460). Only tests/ and bench.py's reference leg use it.
"""
from fractions import Fraction
import math

import numpy as np

from . import ffi

HELD_OUT = 4
_primes = []


def _is_prime(n):
    if n < 2:
        return False
    for sp in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        if n % sp == 0:
            return n == sp
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in (2, 3, 5, 7, 11):  # a deterministic witness set below 2.1e12
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def primes(K):
    """The K largest primes below 2^31, in descending order."""
    c = (_primes[-1] - 2) if _primes else (1 << 31) - 1
    while len(_primes) < K:
        if _is_prime(c):
            _primes.append(c)
        c -= 2
    return np.array(_primes[:K], dtype=np.uint32)


def z_fraction(z):
    f = Fraction(z).limit_denominator(1 << 20)
    if float(f) != z:
        raise ValueError(f"z = {z!r} is not a small rational")
    return f.numerator, f.denominator


def _reconstruct(u, m):
    """The fraction a/b with a = u b (mod m), |a|, b <= sqrt(m/2), or None
    (half-extended Euclid on (m, u))."""
    bound = math.isqrt(m // 2)
    r0, r1, t0, t1 = m, u % m, 0, 1
    while r1 > bound:
        qq = r0 // r1
        r0, r1 = r1, r0 - qq * r1
        t0, t1 = t1, t0 - qq * t1
    if t1 == 0 or abs(t1) > bound or math.gcd(r1, abs(t1)) != 1:
        return None
    return Fraction(r1, t1)  # Fraction normalises the sign


def ratio(num, den, ok, ps):
    """Exact num/den from residues modulo ps: a Fraction, "inf" where den is
    zero modulo every usable prime, None where the primes do not determine
    it (too few, or a held-out prime disagrees)."""
    if not ok.any():
        return None
    use = np.nonzero(ok & (den != 0))[0]
    if len(use) == 0:
        return "inf"
    if len(use) < HELD_OUT + 2:
        return None
    fit, held = use[:-HELD_OUT], use[-HELD_OUT:]
    X, M = 0, 1
    for k in fit:
        pk = int(ps[k])
        uk = int(num[k]) * pow(int(den[k]), -1, pk) % pk
        X += M * ((uk - X) * pow(M % pk, -1, pk) % pk)
        M *= pk
    fr = _reconstruct(X, M)
    if fr is None:
        return None
    for k in held:
        pk = int(ps[k])
        if (fr.numerator * int(den[k]) - int(num[k]) * fr.denominator) % pk:
            return None
    return fr


def exact_ratios(p, q, z, records, N, h, pairs=None, K0=256, K_max=4096, threads=0):
    """Exact snapshot ratios per trajectory: a list of three Fractions (or
    "inf"), or None where the exact walk is singular or K_max primes do not
    determine them. The prime set grows by doubling; residues of primes
    already walked are kept."""
    zn, zd = z_fraction(z)
    n = len(records)
    out = [None] * n
    todo = list(range(n))
    res = np.zeros((n, 3, 2, 0), dtype=np.uint32)
    ok = np.zeros((n, 0), dtype=bool)
    K = 0
    want = K0
    while todo and want <= K_max:
        ps = primes(want)
        sub = np.asarray(todo)
        r_new, ok_new = ffi.exact_residues(p, q, zn, zd, N, h, records[sub], ps[K:want],
                                           None if pairs is None else np.asarray(pairs)[sub], threads)
        r_all = np.zeros((n, 3, 2, want), dtype=np.uint32)
        o_all = np.zeros((n, want), dtype=bool)
        r_all[:, :, :, :K] = res
        o_all[:, :K] = ok
        r_all[sub, :, :, K:] = r_new
        o_all[sub, K:] = ok_new
        res, ok, K = r_all, o_all, want
        left = []
        for t in todo:
            if not ok[t].any():
                continue  # singular for every prime: the exact walk is invalid
            rs = [ratio(res[t, s, 0], res[t, s, 1], ok[t], ps) for s in range(3)]
            if any(r is None for r in rs):
                left.append(t)
            else:
                out[t] = rs
        todo = left
        want *= 2
    return out


def estimator(rs, method):
    """The reference's estimate on exact ratios r1, r2, r3 (depths N-2h,
    N-h, N): Aitken's r3 - (r2 - r3)^2 / (r1 - 2 r2 + r3) for method 1, the
    raw r3 for method 0 (cmf_pfq.cuh:385-460); None where undefined. A walk
    whose ratios have stopped moving (r1 = r2 = r3, second difference 0) has
    Aitken's value r3, its limit as the differences vanish."""
    if rs is None or any(r == "inf" for r in rs):
        return None
    r1, r2, r3 = rs
    if method == 1:
        den = r1 - 2 * r2 + r3
        if den == 0:
            return r3 if r2 == r3 else None
        return r3 - (r2 - r3) ** 2 / den
    return r3


def verify(p, q, z, records, results, limit_src, N, h, rtol=1e-10, K0=256, threads=0):
    """Rows whose limit is within rtol (relative) of the exact value of its
    own estimator. Returns {"verified": bool[n], "rel_err": float[n] (nan
    where not comparable), "exact_limit": float[n]}."""
    n = len(records)
    src = np.asarray(limit_src)
    valid = (np.asarray(results["valid"]) == 1) & (src >= 0)
    idx = np.nonzero(valid)[0]
    verified = np.zeros(n, dtype=bool)
    rel = np.full(n, np.nan)
    exact = np.full(n, np.nan)
    if len(idx):
        rats = exact_ratios(p, q, z, records[idx], N, h, pairs=src[idx] & 0xFFF, K0=K0, threads=threads)
        for rs, t in zip(rats, idx):
            L = estimator(rs, (int(src[t]) >> 12) & 1)
            if L is None:
                continue
            try:
                exact[t] = float(L)
            except OverflowError:
                exact[t] = math.inf if L > 0 else -math.inf
            lf = float(results["limit"][t])
            if not math.isfinite(lf):
                continue
            err = abs(lf) if L == 0 else abs(Fraction(lf) - L) / abs(L)
            rel[t] = float(err) if err < 1e300 else math.inf
            verified[t] = rel[t] <= rtol
    return {"verified": verified, "rel_err": rel, "exact_limit": exact}
