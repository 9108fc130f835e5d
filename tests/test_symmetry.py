"""Alpha<->beta exchange-symmetry projection of the Davidson corrections (params.symmetry, default on
when the alpha and beta lists are identical and the start is the HF determinant).

The projection t <- (t + t^T)/2 runs over 32 x 32 tile pairs, with 16-byte row accesses when the
string count is a multiple of 16 / sizeof(element) and scalar ones otherwise; the cases below take
both (924 strings: 16-byte path in FP32 and FP64; 923: scalar path).  H commutes with the exchange
and the HF start is symmetric, so a solve with the projection reaches the energy of a solve without
it, and its vector is exchange-symmetric: W[Ia, Ib] = s * W[Ib, Ia] with s the reference's
reordering sign of the two determinants (the library returns W in the reference convention)."""
import numpy as np
import pytest


def _solve(prob, precision, symmetry):
    import sbd_tpb
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    # FP32 vectors stall near |r| ~ 5e-6 on this full-CI-like space, so the mixed solves stop at 1e-5
    eps = 1e-7 if precision == sbd_tpb.FP64 else 1e-5
    p = sbd_tpb.default_params(max_it=20, max_nb=10, eps=eps, precision=precision, symmetry=symmetry)
    r = h.davidson(p, want_vector=True)
    h.close()
    return r


@pytest.mark.gpu
@pytest.mark.parametrize("nstrings", [924, 923])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_gpu_symmetry_projection(nstrings, prec):
    import pyoracle
    import sbd_tpb
    import synth
    prob = synth.make_problem("fci12", nstrings=nstrings)
    precision = sbd_tpb.FP64 if prec == "fp64" else sbd_tpb.MIXED
    on = _solve(prob, precision, 1)
    off = _solve(prob, precision, 0)
    assert on["converged"] and off["converged"]
    # energies are <W|H|W> in FP64: errors of order |r|^2 below these bounds
    tol = 1e-9 if prec == "fp64" else 1e-7
    assert on["energy"] == pytest.approx(off["energy"], abs=tol)
    n, L = len(prob.astr), prob.norb
    W = on["W"].reshape(n, n)
    # reordering sign (-1)^#{(p in Ia, q in Ib): q < p}, checked against the oracle on a sample
    bits = lambda s: ((s[:, None] >> np.arange(L, dtype=np.uint64)) & np.uint64(1)).astype(np.int64)
    lower = np.tril(np.ones((L, L), np.int64), -1)  # [p, q] = 1 for q < p
    sign = 1.0 - 2.0 * ((bits(prob.astr) @ lower @ bits(prob.bstr).T) & 1)
    rng = np.random.default_rng(5)
    for i, j in rng.integers(0, n, size=(50, 2)):
        assert sign[i, j] == pyoracle.reorder_sign(int(prob.astr[i]), int(prob.bstr[j]))
    Ws = W * sign  # the library's internal (separated) convention, in which C = C^T
    assert np.abs(Ws - Ws.T).max() < (1e-12 if prec == "fp64" else 1e-6)
    assert abs(np.linalg.norm(W) - 1.0) < 1e-6
