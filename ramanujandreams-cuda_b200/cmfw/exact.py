"""Exact verification of floating-point walk results.

The GPU exact walk (cmfw_exact_residues) keeps the walk product as rational
residues modulo K primes. The residues of two entries of one column at the
three snapshot depths become exact rationals on the device
(cmfw_exact_reconstruct: per prime the ratio a * b^-1, Garner's
Chinese remaindering with a warp lane per prime, rational reconstruction to
Wang's half-extended-Euclid bound sqrt(P/2), checked against held-out
primes); the host only turns the resulting words into Python integers. A
reconstruction that the primes do not determine is retried on a longer
prefix of the walked primes, then with four times the primes walked.

"Verified" means: the floating-point walk is valid, the exact walk is valid,
and the reported limit agrees with the exact value of the same estimator
(the same matrix ratio, Aitken or raw) within the stated relative tolerance.
"""
from fractions import Fraction
import math

import numpy as np

from . import api

CHECK_PRIMES = 4
_prime_cache = []


def _is_prime_u32(n):
    if n < 2:
        return False
    for sp in (2, 3, 5, 7, 11, 13):
        if n % sp == 0:
            return n == sp
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in (2, 3, 5, 7):  # deterministic below 3.2e9
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


def primes_below_2_31(K):
    """The K largest primes below 2^31, descending."""
    if len(_prime_cache) < K:
        c = (_prime_cache[-1] - 2) if _prime_cache else (1 << 31) - 1
        while len(_prime_cache) < K:
            if _is_prime_u32(c):
                _prime_cache.append(c)
            c -= 2
    return np.array(_prime_cache[:K], dtype=np.uint64)


def _vec_pow(b, e, p):
    """b^e mod p elementwise (uint64 arrays, p < 2^31)."""
    r = np.ones_like(b)
    b = b % p
    e = e.copy()
    while np.any(e):
        odd = (e & 1).astype(bool)
        r = np.where(odd, (r * b) % p, r)
        b = (b * b) % p
        e >>= 1
    return r


def _rational_reconstruct(u, m):
    """a/b with a = u*b mod m, |a|, b <= sqrt(m/2), or None."""
    bound = math.isqrt(m // 2)
    r0, r1 = m, u % m
    t0, t1 = 0, 1
    while r1 > bound:
        qq = r0 // r1
        r0, r1 = r1, r0 - qq * r1
        t0, t1 = t1, t0 - qq * t1
    if t1 == 0 or abs(t1) > bound or math.gcd(r1, abs(t1)) != 1:
        return None
    if t1 < 0:
        r1, t1 = -r1, -t1
    return Fraction(r1, t1)


def _ratio_from_residues(a, b, ok, primes):
    """Exact a/b from residues a[K], b[K] modulo `primes`.

    Returns a Fraction, "inf" when b vanishes modulo every surviving prime
    (b == 0 exactly), or None when the primes do not determine the value
    (too few, or the reconstruction fails the held-out check).
    """
    p = primes
    usable = ok & (b != 0)
    if not ok.any():
        return None
    if not usable.any():
        return "inf"
    use = np.nonzero(usable)[0]
    if len(use) < CHECK_PRIMES + 2:
        return None
    bi = _vec_pow(b.astype(np.uint64), p - 2, p)
    u = (a.astype(np.uint64) * bi) % p
    crt, chk = use[:-CHECK_PRIMES], use[-CHECK_PRIMES:]
    X, M = 0, 1
    for k in crt:  # incremental Chinese remaindering
        pk, uk = int(p[k]), int(u[k])
        X += M * (((uk - X) * pow(M % pk, -1, pk)) % pk)
        M *= pk
    fr = _rational_reconstruct(X, M)
    if fr is None:
        return None
    for k in chk:
        pk = int(p[k])
        if (fr.numerator - int(u[k]) * fr.denominator) % pk != 0:
            return None
    return fr


def exact_ratios(desc, records, N, h, pairs=None, K0=64, K_max=4096):
    """Exact snapshot ratios M[i][c]/M[j][c] at N-2h, N-h, N per trajectory.

    Returns (ratios, K_used): ratios[t] is a list of three Fractions ("inf"
    where the denominator is exactly zero), or None where the exact walk is
    invalid (a divisor vanished for every prime).
    """
    torch = api._torch()
    n = len(records)
    ratios = [None] * n
    K_used = np.zeros(n, dtype=np.int64)
    todo = np.arange(n)
    K_run = K0
    while len(todo) and K_run <= K_max:
        # one exact walk with K_run primes; reconstructions on growing prefixes
        primes = primes_below_2_31(K_run)
        sub = records[todo]
        sub_pairs = None if pairs is None else np.asarray(pairs)[todo]
        d_in = api.to_device(sub)
        d_res, d_ok, d_primes = api.exact_residues_device(desc, d_in, len(sub), N, h, primes, sub_pairs)
        pending = np.arange(len(todo))
        K = min(64, K_run)
        while len(pending):
            sel = torch.from_numpy(pending).cuda()
            st, fr = api.exact_reconstruct(d_res[sel].contiguous(), d_ok[sel].contiguous(), d_primes,
                                           len(pending), K)
            left = []
            for r, li in enumerate(pending):
                t = todo[li]
                if (st[r] == 3).all():
                    ratios[t] = None  # singular for every prime: the exact walk is invalid
                    K_used[t] = K
                elif (st[r] == 2).any():
                    left.append(li)
                else:
                    ratios[t] = ["inf" if st[r, k] == 1 else Fraction(*fr[r][k]) for k in range(3)]
                    K_used[t] = K
            pending = np.array(left, dtype=np.int64)
            if K >= K_run:
                break
            K = min(K * 2, K_run)
        todo = todo[pending] if len(pending) else np.zeros(0, dtype=np.int64)
        K_run *= 4
    for t in todo:
        K_used[t] = -1  # not determined within K_max primes
    return ratios, K_used


def exact_estimator(rs, method):
    """The limit estimator of the reference's reduction on exact ratios."""
    if rs is None or any(r == "inf" for r in rs):
        return None
    r1, r2, r3 = rs
    if method == 1:
        den = r1 - 2 * r2 + r3
        if den != 0:
            return r3 - (r2 - r3) ** 2 / den
    return r3


def rounding_floor(rs, method, u=2.0 ** -51):
    """The estimator's relative change when each exact ratio moves by a
    relative u (4 units of 2^-53 by default): the error that computing the
    ratios in double precision alone can leave in the limit, however exact
    the walk. Aitken's estimator divides by a second difference of the
    ratios, so on partially converged walks this floor reaches 1e-10 and
    beyond. None where the estimator has no exact value.

    Worked in floating point from the exact differences D = r2 - r3 and
    E = r1 - 2 r2 + r3 (exact, then rounded), so that the perturbed
    estimate's change is formed from the small increments themselves:
    dL = e3 r3 - ((2 D dD + dD^2) E - D^2 dE) / (E (E + dE)) with
    dD = e2 r2 - e3 r3, dE = e1 r1 - 2 e2 r2 + e3 r3, e_i = +-u."""
    L = exact_estimator(rs, method)
    if L is None or L == 0:
        return None
    r1, r2, r3 = rs
    Lf = abs(float(L))
    f1, f2, f3 = float(r1), float(r2), float(r3)
    if method != 1 or r1 - 2 * r2 + r3 == 0:
        return float(u * abs(f3) / Lf)
    D, E = float(r2 - r3), float(r1 - 2 * r2 + r3)
    if E == 0.0 or not math.isfinite(E) or not math.isfinite(D):
        return math.inf  # the second difference is below the double range: no usable floor
    worst = 0.0
    for e1 in (-u, u):
        for e2 in (-u, u):
            for e3 in (-u, u):
                dD = e2 * f2 - e3 * f3
                dE = e1 * f1 - 2.0 * e2 * f2 + e3 * f3
                if E + dE == 0.0:
                    # the moved second difference vanishes: the estimate falls back to r3
                    dL = (f3 * (1.0 + e3)) - float(L)
                else:
                    dL = e3 * f3 - ((2.0 * D * dD + dD * dD) * E - D * D * dE) / (E * (E + dE))
                worst = max(worst, abs(dL) / Lf)
    return float(worst)


def verify(desc, records, results, limit_src, N, h, rtol=1e-10, K0=1024):
    """Per-trajectory exact check of float results.

    Returns a dict of arrays: verified (bool), rel_err (float, nan where not
    comparable), exact_limit (float), K (primes used), floor (float: the
    rounding_floor of the trajectory's estimator, nan where undefined).
    """
    n = len(records)
    valid = np.asarray(results["valid"]) == 1
    src = np.asarray(limit_src)
    idx = np.nonzero(valid & (src >= 0))[0]
    verified = np.zeros(n, dtype=bool)
    rel = np.full(n, np.nan)
    exact_limit = np.full(n, np.nan)
    Ks = np.zeros(n, dtype=np.int64)
    floor = np.full(n, np.nan)
    if len(idx):
        ratios, K_used = exact_ratios(desc, records[idx], N, h, pairs=src[idx] & 0xFFF, K0=K0)
        for li, t in enumerate(idx):
            Ks[t] = K_used[li]
            L = exact_estimator(ratios[li], (int(src[t]) >> 12) & 1)
            if L is None:
                continue
            fl = rounding_floor(ratios[li], (int(src[t]) >> 12) & 1)
            floor[t] = np.nan if fl is None else fl
            try:
                exact_limit[t] = float(L)
            except OverflowError:  # beyond the double range: no double is within rtol
                exact_limit[t] = math.inf if L > 0 else -math.inf
            lf = float(results["limit"][t])
            if not math.isfinite(lf):
                err = math.inf
            elif L == 0:
                err = abs(lf)
            else:
                err = abs(Fraction(lf) - L) / abs(L)
            rel[t] = float(err) if err < 1e300 else math.inf
            verified[t] = rel[t] <= rtol
    return {"verified": verified, "rel_err": rel, "exact_limit": exact_limit, "K": Ks, "floor": floor}


def export_topk(desc, records, results, N, h, k=100, K0=1024):
    """Exact rational export of the k valid trajectories with the largest
    finite delta: for each, the ratio p/q = M[0][r-1] / M[1][r-1] at depths
    N-2h, N-h and N as exact rationals (numerator and denominator as decimal
    strings), beside the floating-point limit and delta -- the input an exact
    refinement of the most promising candidates starts from."""
    delta = np.asarray(results["delta"], float)
    ok = (np.asarray(results["valid"]) == 1) & np.isfinite(delta)
    idx = np.nonzero(ok)[0]
    idx = idx[np.argsort(-delta[idx], kind="stable")][:k]
    entries = []
    if len(idx) == 0:
        return entries
    ratios, K_used = exact_ratios(desc, records[idx], N, h, K0=K0)
    p, q = desc.p, desc.q
    for li, t in enumerate(idx):
        rs = ratios[li]
        e = {"index": int(t), "dir": [int(x) for x in records["dir"][t][:p + q]],
             "start": [float(x) for x in records["start"][t][:p + q]],
             "delta": float(delta[t]), "limit": float(results["limit"][t]), "primes": int(K_used[li])}
        if rs is None:
            e["exact"] = None
        else:
            e["exact"] = [None if r == "inf" else {"depth": d, "num": str(r.numerator), "den": str(r.denominator)}
                          for r, d in zip(rs, (N - 2 * h, N - h, N))]
        entries.append(e)
    return entries
