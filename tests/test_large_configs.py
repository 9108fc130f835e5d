"""The benchmark's selected-CI workloads pinned to the reference: norb=24 with 4,000 x 4,000 strings
(16M determinants), norb=28 with 10,000 x 10,000 strings (100M, the learned-preconditioner config) and
norb=32 with 20,000 x 20,000 strings (400M determinants, the benchmark's workload), same seeded
generators as bench.py.

The fixtures sci24.npz / sci28.npz / sci32.npz come from the reference's own code (oracle/_ref/ref_dump, made by
tests/golden/make_golden.py): its excitation tables (MakeHelpers + RemakeHelpers, tpb/helper.h:
710-1226), H_ii (makeQChamDiagTerms, tpb/qcham.h:290-340) and one sigma (mult, tpb/mult.h:625-881) of
the closed-form vector x_i = ((i * 0x9E3779B97F4A7C15 mod 2^64) >> 11) / 2^53 - 1/2, stored as 512
sampled entries plus sum / sum of squares / sum of |.| over all N; the 16M set also holds the
reference's FP64 Davidson energy (tpb/davidson.h:667-930).  The closed form lets every check
regenerate the input at full size without storing it.  The 16M and 100M sets also hold the reference's
FP64 Davidson energy from the HF start.

CPU: the oracle's tables and its sigma at the sampled determinants equal the reference's.
GPU: the library's tables are bit-exact, H_ii and sigma match at the samples (1e-12 of the largest
sampled |sigma|) and in the whole-vector sums, sigma matches the oracle at 256 more determinants, and
at 16M and 100M determinants the FP64 Davidson energy is within 1e-8 Ha of the reference's, the mixed
one within 1e-6 Ha.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_cases

CASES = [c for c in ("sci24", "sci28", "sci32") if os.path.exists(os.path.join(GOLDEN, f"{c}.npz"))]
K = 0x9E3779B97F4A7C15


def _fixture(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz"))), golden_cases()[name]


def _reference_tables(g):
    """(kind -> (off, ket, cran)) as the reference wrote them; beta = alpha strings, labels + 1."""
    t = {}
    for k, k0, shift in (("sa", "sa", 0), ("da", "da", 0), ("sb", "sa", 1), ("db", "da", 1)):
        t[k] = (g[f"t0_{k0}_off"], g[f"t0_{k0}_ket"].astype(np.uint64), g[f"t0_{k0}_cran"].astype(np.int32) + shift)
    return t


@pytest.fixture(scope="module", params=CASES)
def case(request):
    import synth
    name = request.param
    g, meta = _fixture(name)
    prob = synth.make_problem(name)
    assert np.array_equal(prob.astr, g["astr"]) and np.array_equal(prob.bstr, g["bstr"])
    assert g["tables_deduped"][0] == 1
    return name, prob, g, meta


def test_hash_vector_regenerates_reference_input(case):
    import pyoracle
    name, prob, g, meta = case
    assert np.array_equal(pyoracle.hash_vector(g["idx"]), g["sigma_in_sample"])


def test_oracle_matches_reference(case, oracle):
    name, prob, g, meta = case
    ham = oracle.Hamiltonian.from_arrays(prob.norb, prob.nelec, prob.core, prob.h1, prob.eri_packed)
    sysm = oracle.System(ham, prob.astr, prob.bstr)
    for k, (off, ket, cran) in _reference_tables(g).items():
        o, kk, c = sysm.table(k)
        assert np.array_equal(o, off) and np.array_equal(kk, ket) and np.array_equal(c, cran), k
    s = sysm.sigma_rows(g["idx"])
    ref = g["sigma_out_sample"]
    assert np.max(np.abs(s - ref)) <= 1e-13 * np.max(np.abs(ref))


def _hash_vector_device(n):
    import torch
    i = torch.arange(n, dtype=torch.int64, device="cuda")
    i.mul_(K - (1 << 64))  # wraps modulo 2^64 in two's complement, as the unsigned product
    i.bitwise_right_shift_(11).bitwise_and_((1 << 53) - 1)
    x = i.double()
    del i
    return x.mul_(2.0 ** -53).sub_(0.5)


@pytest.mark.gpu
def test_gpu_matches_reference(case, oracle):
    import torch

    import sbd_tpb
    name, prob, g, meta = case
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    ref = _reference_tables(g)
    for kind, k in ((sbd_tpb.SINGLES_ALPHA, "sa"), (sbd_tpb.DOUBLES_ALPHA, "da"),
                    (sbd_tpb.SINGLES_BETA, "sb"), (sbd_tpb.DOUBLES_BETA, "db")):
        off, ket, cran = h.table(kind)
        assert np.array_equal(off, ref[k][0]) and np.array_equal(ket, ref[k][1]), k
        assert np.array_equal(cran, ref[k][2]), k
    idx = torch.from_numpy(g["idx"].astype(np.int64)).cuda()
    hii = h.diagonal_device()
    hs = hii[idx].cpu().numpy()
    assert np.max(np.abs(hs - g["hii_sample"])) <= 1e-13 * np.max(np.abs(g["hii_sample"]))
    del hii
    x = _hash_vector_device(prob.ndet)
    assert np.array_equal(x[idx].cpu().numpy(), g["sigma_in_sample"])
    y = torch.empty_like(x)
    h.sigma_device(x, y, separated=False)  # reference sign convention and order
    del x
    ys = y[idx].cpu().numpy()
    refs = g["sigma_out_sample"]
    scale = np.max(np.abs(refs))
    assert np.max(np.abs(ys - refs)) <= 1e-12 * scale
    sums = np.array([float(y.sum()), float((y * y).sum()), float(y.abs().sum())])
    assert np.allclose(sums, g["sigma_out_sum"], rtol=1e-10, atol=1e-10 * scale), (sums, g["sigma_out_sum"])
    # and the oracle at 256 other determinants
    rows = np.random.default_rng(17).integers(0, prob.ndet, 256)
    ham = oracle.Hamiltonian.from_arrays(prob.norb, prob.nelec, prob.core, prob.h1, prob.eri_packed)
    orc = oracle.System(ham, prob.astr, prob.bstr).sigma_rows(rows)
    got = y[torch.from_numpy(rows.astype(np.int64)).cuda()].cpu().numpy()
    assert np.max(np.abs(got - orc)) <= 1e-12 * np.max(np.abs(orc))
    del y
    if "energy" in meta:
        it, nb, tol = meta["davidson"]
        r = h.davidson(sbd_tpb.default_params(max_it=it, max_nb=nb, eps=tol), want_vector=False)
        assert abs(r["energy"] - meta["energy"]) < 1e-8, (r["energy"], meta["energy"])
        rm = h.davidson(sbd_tpb.default_params(max_it=it, max_nb=8, eps=1e-5, precision=sbd_tpb.MIXED),
                        want_vector=False)
        assert abs(rm["energy"] - meta["energy"]) < 1e-6, (rm["energy"], meta["energy"])
    h.close()
