"""The device reconstruction of exact ratios (cmfw_exact_reconstruct,
marked gpu): Garner CRT with a lane per prime, rational reconstruction to
Wang's bound and the held-out check, against Python integers -- synthetic
fractions of every size (never a wrong value: too few primes give
"undetermined"), the exact zero and singular cases, and the GPU exact
walk's own residues against the host reconstruction."""
from fractions import Fraction

import numpy as np
import pytest

import cmfw
import cmfw.workloads as wl
from cmfw import api, exact

pytestmark = pytest.mark.gpu


def _upload(res, ok, primes):
    import torch
    return (torch.from_numpy(np.ascontiguousarray(res).view(np.int32)).cuda(),
            torch.from_numpy(np.ascontiguousarray(ok, dtype=np.uint8)).cuda(),
            torch.from_numpy(np.ascontiguousarray(primes, dtype=np.uint32).view(np.int32)).cuda())


def _residues(fr, ps):
    a = np.array([fr.numerator % int(p) for p in ps], dtype=np.uint32)
    b = np.array([fr.denominator % int(p) for p in ps], dtype=np.uint32)
    return a, b


def test_synthetic_fractions_of_every_size(cuda):
    rng = np.random.default_rng(7)
    K = 256
    ps = exact.primes_below_2_31(K).astype(np.uint32)
    cases = []
    for bits in (1, 20, 61, 200, 1000, 2500, 3700, 3900, 4100, 6000):
        for _ in range(3):
            num = int(rng.integers(1, 2 ** 62)) << max(0, bits - 62) | int(rng.integers(0, 2 ** 31))
            num = num % (1 << bits) + (1 << (bits - 1)) if bits > 1 else 1
            den = (int(rng.integers(1, 2 ** 62)) << max(0, bits - 62)) % (1 << bits) + 1
            sign = -1 if rng.random() < 0.5 else 1
            cases.append(Fraction(sign * num, den))
    cases.append(Fraction(0))
    n = (len(cases) + 2) // 3
    cases += [Fraction(1)] * (3 * n - len(cases))
    res = np.zeros((n, 3, 2, K), dtype=np.uint32)
    ok = np.ones((n, K), dtype=np.uint8)
    for i, fr in enumerate(cases):
        res[i // 3, i % 3, 0], res[i // 3, i % 3, 1] = _residues(fr, ps)
    ok[0, 5] = 0  # an unusable prime is skipped
    d_res, d_ok, d_ps = _upload(res, ok, ps)
    for Kp in (64, 128, 256):
        st, frs = api.exact_reconstruct(d_res, d_ok, d_ps, n, Kp)
        for i, fr in enumerate(cases):
            row = i // 3
            usable = [int(p) for k, p in enumerate(ps[:Kp]) if ok[row, k]]
            P = 1
            for p in usable[:-4]:
                P *= p
            Lb = (P.bit_length() - 2) // 2
            s = st[row, i % 3]
            assert s in (0, 2), (i, s)
            if s == 0:  # never a wrong value
                assert Fraction(*frs[row][i % 3]) == fr, (i, Kp)
            # within Wang's bounds the reconstruction must succeed
            if abs(fr.numerator) < (1 << Lb) and fr.denominator.bit_length() + Lb + 1 <= P.bit_length() - 1:
                assert s == 0, (i, Kp, fr.numerator.bit_length(), fr.denominator.bit_length(), P.bit_length())
        assert (st == 0).sum() >= 6 and (st == 2).sum() >= 3


def test_zero_denominator_and_singular(cuda):
    K = 64
    ps = exact.primes_below_2_31(K).astype(np.uint32)
    res = np.zeros((2, 3, 2, K), dtype=np.uint32)
    ok = np.ones((2, K), dtype=np.uint8)
    res[0, :, 0] = 5  # denominator residues all zero: an exact zero denominator
    ok[1] = 0         # no usable prime
    d_res, d_ok, d_ps = _upload(res, ok, ps)
    st, _ = api.exact_reconstruct(d_res, d_ok, d_ps, 2, K)
    assert (st[0] == 1).all() and (st[1] == 3).all()


def test_device_reconstruction_matches_the_host_on_walk_residues(cuda):
    recs = wl.zeta_directions(6, 5, 3000, 20261203)
    desc = cmfw.make_desc(6, 5, 1.0)
    out, src = cmfw.walk("f64", desc, recs, 1000, 50, with_limit_src=True)
    sub = recs[out["valid"] == 1][:10]
    K = 1024
    ps = exact.primes_below_2_31(K)
    res, ok = cmfw.exact_residues(desc, sub, 1000, 50, ps.astype(np.uint32))
    d_res, d_ok, d_ps = _upload(res, ok, ps.astype(np.uint32))
    st, frs = api.exact_reconstruct(d_res, d_ok, d_ps, len(sub), K)
    for t in range(len(sub)):
        for s in range(3):
            host = exact._ratio_from_residues(res[t, s, 0], res[t, s, 1], ok[t], ps)
            if host is None:
                assert st[t, s] == 2
            elif host == "inf":
                assert st[t, s] == 1
            else:
                assert st[t, s] == 0 and Fraction(*frs[t][s]) == host
    assert (st == 0).sum() >= 15
