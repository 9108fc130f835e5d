"""The separated sign convention the GPU path uses, checked against the reference's formulas.

The reference evaluates every element on the interleaved determinant (basic/determinants.h:97-142,
230-501).  The library works with all alpha creators ordered before all beta creators, where
H_sep = D H_ref D, D = diag((-1)^#{(p in Ia, q in Ib): q < p}); this test builds H_sep from the
one-spin formulas the kernels use and compares it with the oracle's interleaved elements.
"""
import itertools

import numpy as np

from conftest import golden_problem


def _popc(x):
    return bin(int(x)).count("1")


def _bits(x):
    return [p for p in range(64) if (int(x) >> p) & 1]


def _par_open(s, a, b):
    lo, hi = min(a, b), max(a, b)
    m = ((1 << hi) - 1) & ~((2 << lo) - 1)
    return -1 if _popc(int(s) & m) & 1 else 1


def _above_parity_mask(a):
    s = int(a)
    for k in (1, 2, 4, 8, 16, 32):
        s ^= s >> k
    return s >> 1


def h_sep(eri, h1, Ia, Ib, Ja, Jb):
    da, db = _popc(int(Ia) ^ int(Ja)), _popc(int(Ib) ^ int(Jb))

    def single(I, J, other):
        cr = _bits(int(I) & ~int(J))[0]
        an = _bits(int(J) & ~int(I))[0]
        v = h1[an, cr] + sum(eri[an, cr, j, j] - eri[an, j, j, cr] for j in _bits(I))
        v += sum(eri[an, cr, k, k] for k in _bits(other))
        return _par_open(I, cr, an) * v

    def double(I, J):
        cr, an = _bits(int(I) & ~int(J)), _bits(int(J) & ~int(I))
        i0, j0, a0, b0 = cr[0], cr[1], an[0], an[1]
        s = _par_open(I, i0, a0) * _par_open(I, j0, b0) * (-1 if (a0 > j0 or b0 < i0) else 1)
        return s * (eri[a0, i0, b0, j0] - eri[a0, j0, b0, i0])

    if da == 2 and db == 0:
        return single(Ia, Ja, Ib)
    if da == 0 and db == 2:
        return single(Ib, Jb, Ia)
    if da == 4 and db == 0:
        return double(Ia, Ja)
    if da == 0 and db == 4:
        return double(Ib, Jb)
    if da == 2 and db == 2:
        cra, ana = _bits(int(Ia) & ~int(Ja))[0], _bits(int(Ja) & ~int(Ia))[0]
        crb, anb = _bits(int(Ib) & ~int(Jb))[0], _bits(int(Jb) & ~int(Ib))[0]
        return _par_open(Ia, cra, ana) * _par_open(Ib, crb, anb) * eri[cra, ana, crb, anb]
    return None


def test_reorder_sign_mask(oracle):
    rng = np.random.default_rng(5)
    for _ in range(2000):
        a, b = int(rng.integers(0, 1 << 40)), int(rng.integers(0, 1 << 40))
        d = -1 if _popc(_above_parity_mask(a) & b) & 1 else 1
        assert d == oracle.reorder_sign(a, b)


def test_h_ref_equals_d_hsep_d(oracle):
    import synth
    prob, g, meta = golden_problem("syn10_ab")
    L = prob.norb
    eri = synth.unpack_eri(prob.eri_packed, L)
    ham = oracle.Hamiltonian.from_arrays(L, prob.nelec, prob.core, prob.h1, prob.eri_packed)
    s = oracle.System(ham, prob.astr, prob.bstr)
    rng = np.random.default_rng(1)
    A = prob.astr[rng.choice(len(prob.astr), 24, replace=False)]
    B = prob.bstr[rng.choice(len(prob.bstr), 18, replace=False)]
    worst, count = 0.0, 0
    for Ia, Ib, Ja, Jb in itertools.product(A, B, A, B):
        v = h_sep(eri, prob.h1, Ia, Ib, Ja, Jb)
        if v is None:
            continue
        ref = s.hij(Ja, Jb, Ia, Ib)  # Hij evaluates on its second determinant, the bra
        d = oracle.reorder_sign(Ia, Ib) * oracle.reorder_sign(Ja, Jb)
        worst = max(worst, abs(ref - d * v))
        count += 1
    assert count > 1000
    assert worst < 1e-13
