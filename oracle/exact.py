"""Exact rational walk with Python Fractions -- TEST INFRASTRUCTURE.

The same lattice path, column and update as the reference
(cmf_pfq.cuh:127-322) with no normalisation and no rounding: every entry of
the walk matrix is an exact rational. Used to check the GPU exact walk's
residues and the floating-point walks' error on small cases (it runs in
seconds only for N up to a few hundred).
"""
from fractions import Fraction


def rank_of(p, q, z):
    r = max(p, q + 1)
    return r - 1 if (Fraction(z) == 1 and p == q + 1) else r


def _theta_product(vals):
    out = [Fraction(1)]
    for v in vals:
        nxt = [Fraction(0)] * (len(out) + 1)
        for k, c in enumerate(out):
            nxt[k] += c * v
            nxt[k + 1] += c
        out = nxt
    return out


def column(pos, p, q, z, dim):
    """-d[i]/lead of D(theta) at `pos` (cmf_pfq.cuh:146-181); None if lead == 0."""
    px = _theta_product(pos[:p])
    py = _theta_product([y - 1 for y in pos[p:p + q]])
    d = [Fraction(0)] * (max(p, q + 1) + 1)
    for k in range(p + 1):
        d[k] = -z * px[k]
    for k in range(q + 1):
        d[k + 1] += py[k]
    lead = d[dim]
    if lead == 0:
        return None
    return [-d[i] / lead for i in range(dim)]


def _step(M, col, a, inverse, dim):
    """M (I + C/a) or M (I + C/a)^-1 (cmf_pfq.cuh:186-239), exactly."""
    if a == 0:
        return None
    out = []
    for m in M:
        if not inverse:
            dot = sum(m[k] * col[k] for k in range(dim))
            out.append([m[j] + m[j + 1] / a for j in range(dim - 1)] + [m[dim - 1] + dot / a])
        else:
            al = [Fraction(0)] * dim
            be = [Fraction(0)] * dim
            be[dim - 1] = Fraction(1)
            for j in range(dim - 2, -1, -1):
                al[j] = m[j] - al[j + 1] / a
                be[j] = -be[j + 1] / a
            da = sum(al[k] * col[k] for k in range(dim))
            db = sum(be[k] * col[k] for k in range(dim))
            sd = 1 + db / a
            if sd == 0:
                return None
            t = (m[dim - 1] - da / a) / sd
            out.append([al[j] + be[j] * t for j in range(dim)])
    return out


def walk(p, q, z, start, direction, N, snapshots=()):
    """Exact walk. Returns (matrix after N steps or None if singular,
    {step: matrix} for the requested snapshot steps)."""
    z = Fraction(z)
    dim = rank_of(p, q, z)
    M = [[Fraction(int(i == j)) for j in range(dim)] for i in range(dim)]
    pos = [Fraction(v) for v in start[:p + q]]
    d = list(direction[:p + q])
    naxes = p + q
    mx = max(abs(x) for x in d) if d else 0
    snaps = {}
    for step in range(1, N + 1):
        for level in range(mx, 0, -1):
            for ax in range(naxes - 1, -1, -1):
                if abs(d[ax]) < level:
                    continue
                sg = 1 if d[ax] > 0 else -1
                ev = list(pos)
                if ax < p:
                    inverse = sg < 0
                    a = pos[ax] if sg > 0 else pos[ax] - 1
                    if inverse:
                        ev[ax] -= 1
                else:
                    inverse = sg > 0
                    a = pos[ax] if sg > 0 else pos[ax] - 1
                    if inverse:
                        ev[ax] += 1
                col = column(ev, p, q, z, dim)
                if col is None:
                    return None, snaps
                M = _step(M, col, a, inverse, dim)
                if M is None:
                    return None, snaps
                pos[ax] += sg
        if step in snapshots:
            snaps[step] = [row[:] for row in M]
    return M, snaps


def residue(fr, prime):
    """An exact rational modulo a prime (its denominator must be invertible)."""
    return fr.numerator * pow(fr.denominator, -1, prime) % prime
