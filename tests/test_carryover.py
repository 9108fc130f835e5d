"""Carry-over strings (tpb/sbdiag.h:690-736).

CPU: the oracle's restatement (orc_string_weights / orc_carryover_select / orc_singles_extend)
against the reference's own CarryOverAdet/Bdet and SinglesExtendHalfdets, run by
oracle/_ref/ref_dump on the fixtures' CI vectors (tests/golden/make_golden.py), plus the
selection rules at their edges.  GPU: the library's carry-over (sbd_tpb_carryover_strings, the
Davidson hook and the CLI flags) against the reference's strings and the oracle, bit-exact on the
strings, 1e-12 on the weights."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden_cases, golden_problem, load_golden

CO_CASES = [n for n, m in golden_cases().items() if "carryover" in m]


def _ref_outputs(g):
    ratio, thr, cut, tw_a, tw_b, total = g["carryover"]
    return ratio, thr, cut, tw_a, tw_b, total


@pytest.mark.parametrize("name", CO_CASES)
def test_oracle_carryover_matches_reference(name):
    import pyoracle
    prob, g, meta = golden_problem(name)
    ratio, thr, cut, tw_a, tw_b, total = _ref_outputs(g)
    W = g["W"]
    co_a, co_b, _, _, _ = pyoracle.carryover(W, prob.astr, prob.bstr, prob.norb, 1, 0.0, thr)
    np.testing.assert_array_equal(co_a, g["co1_a"])
    np.testing.assert_array_equal(co_b, g["co1_b"])
    ra, rb, ta, tb, _ = pyoracle.carryover(W, prob.astr, prob.bstr, prob.norb, 1, ratio, thr)
    np.testing.assert_array_equal(ra, g["co1r_a"])
    np.testing.assert_array_equal(rb, g["co1r_b"])
    assert ta == pytest.approx(tw_a, abs=1e-12) and tb == pytest.approx(tw_b, abs=1e-12)
    if "co2_a" in g:  # the reference extends only equal electron counts (see ref_dump.cc)
        xa, xb, _, _, _ = pyoracle.carryover(W, prob.astr, prob.bstr, prob.norb, 2, 0.0, thr)
        np.testing.assert_array_equal(xa, g["co2_a"])
        np.testing.assert_array_equal(xb, g["co2_b"])
    if "co3_a" in g:
        ya, yb, _, _, t = pyoracle.carryover(W, prob.astr, prob.bstr, prob.norb, 3, 0.0, cut)
        np.testing.assert_array_equal(ya, g["co3_a"])
        np.testing.assert_array_equal(yb, g["co3_b"])
        assert t == pytest.approx(total, abs=1e-12)


def test_oracle_select_edges():
    import pyoracle
    w = np.array([0.1, 0.4, 0.1, 0.3, 0.1])
    # equal weights keep ascending index order
    order, _ = pyoracle.carryover_select(w, 0.0, 0.0)
    np.testing.assert_array_equal(order, [1, 3, 0, 2, 4])
    # running weights 0.4 0.7 0.8 0.9 1.0: with threshold 0.25 the first above 0.75 is the third
    order, _ = pyoracle.carryover_select(w, 0.0, 0.25)
    np.testing.assert_array_equal(order, [1, 3, 0])
    # threshold 0 (running weight never above 1): every string, not one past the end
    order, _ = pyoracle.carryover_select(w / w.sum() * 0.5, 0.0, 0.0)
    assert len(order) == 5
    # ratio: floor(ratio * n) strings and 1 - their weight
    order, t = pyoracle.carryover_select(w, 0.5, 0.01)
    np.testing.assert_array_equal(order, [1, 3])
    assert t == pytest.approx(1.0 - 0.7)
    order, t = pyoracle.carryover_select(w, 0.1, 0.01)
    assert len(order) == 0 and t == pytest.approx(1.0)


def test_oracle_singles_extend_edges():
    import pyoracle
    # a string and its e(L-e) singles; duplicates between strings appear once; ascending order
    s = np.array([0b0011, 0b0101], np.uint64)
    out = pyoracle.singles_extend(s, 4)
    expect = sorted({0b0011, 0b0101, 0b0110, 0b1001, 0b1010, 0b1100, 0b0011 ^ 0b0110 ^ 0b0011})
    assert list(out) == sorted(set(expect) | {0b0101 ^ 0b0001 ^ 0b0010})
    assert len(pyoracle.singles_extend(np.array([(1 << 64) - 1], np.uint64), 64)) == 1
    full = pyoracle.singles_extend(np.array([0b111], np.uint64), 6)
    assert len(full) == 1 + 3 * 3


# ---------------------------------------------------------------------------------------------- GPU


def _handle(prob):
    import sbd_tpb
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    return h


@pytest.mark.gpu
@pytest.mark.parametrize("name", CO_CASES)
def test_gpu_carryover_matches_reference(name):
    import sbd_tpb
    prob, g, meta = golden_problem(name)
    ratio, thr, cut, tw_a, tw_b, total = _ref_outputs(g)
    h = _handle(prob)
    W = g["W"]
    r = h.carryover(W, sbd_tpb.CARRYOVER_DOMINANT, 0.0, thr)
    np.testing.assert_array_equal(r["astr"], g["co1_a"])
    np.testing.assert_array_equal(r["bstr"], g["co1_b"])
    r = h.carryover(W, sbd_tpb.CARRYOVER_DOMINANT, ratio, thr)
    np.testing.assert_array_equal(r["astr"], g["co1r_a"])
    np.testing.assert_array_equal(r["bstr"], g["co1r_b"])
    assert r["truncated_a"] == pytest.approx(tw_a, abs=1e-12)
    assert r["truncated_b"] == pytest.approx(tw_b, abs=1e-12)
    if "co2_a" in g:
        r = h.carryover(W, sbd_tpb.CARRYOVER_DOMINANT_SINGLES, 0.0, thr)
        np.testing.assert_array_equal(r["astr"], g["co2_a"])
        np.testing.assert_array_equal(r["bstr"], g["co2_b"])
    if "co3_a" in g:
        r = h.carryover(W, sbd_tpb.CARRYOVER_CUTOFF_SINGLES, 0.0, cut)
        np.testing.assert_array_equal(r["astr"], g["co3_a"])
        np.testing.assert_array_equal(r["bstr"], g["co3_b"])
        assert r["total_weight"] == pytest.approx(total, abs=1e-12)


@pytest.mark.gpu
def test_gpu_carryover_unequal_counts_against_oracle():
    """Types 2 and 3 with different alpha/beta electron counts (where the reference fails): each
    spin is extended with its own count, as the oracle does."""
    import pyoracle
    prob, g, meta = golden_problem("syn10_ab")
    h = _handle(prob)
    W = g["W"]
    for kind, thr in ((2, 1e-3), (3, 1e-4), (3, 0.0), (2, 0.2)):
        r = h.carryover(W, kind, 0.0, thr)
        oa, ob, _, _, t = pyoracle.carryover(W, prob.astr, prob.bstr, prob.norb, kind, 0.0, thr)
        np.testing.assert_array_equal(r["astr"], oa)
        np.testing.assert_array_equal(r["bstr"], ob)
        if kind == 3:
            assert r["total_weight"] == pytest.approx(t, rel=1e-13)


@pytest.mark.gpu
@pytest.mark.parametrize("na,nb", [(160000, 13), (97, 70001), (2048, 2048)])
def test_gpu_carryover_weights_at_size(na, nb):
    """Shapes that exercise the row sub-bands (more than 256 rows per CTA), ragged column chunks
    and a W larger than one chunk in both directions: selections equal the oracle's on the same
    vector (random amplitudes, so no ties), weights to 1e-12."""
    import pyoracle
    import sbd_tpb
    import synth
    from sbd_tpb import Problem
    rng = np.random.default_rng(na + nb)
    L = 40
    def strings(n, e):
        out = set()
        while len(out) < n:
            out.add(sum(1 << int(p) for p in rng.choice(L, e, replace=False)))
        return np.array(sorted(out), np.uint64)
    h1, eri, core = synth.synthetic_hamiltonian(L, seed=3)
    prob = Problem(norb=L, nelec=10, core=core, h1=h1, eri_packed=eri, astr=strings(na, 5),
                   bstr=strings(nb, 5))
    h = sbd_tpb.Handle(0)
    h.set_problem(prob, build=False)  # carry-over needs the strings only
    W = rng.standard_normal(na * nb) * np.exp(-rng.uniform(0, 12, na * nb))
    W /= np.linalg.norm(W)
    for kind, ratio, thr in ((1, 0.0, 0.05), (1, 0.3, 0.0), (3, 0.0, 1e-9)):
        r = h.carryover(W, kind, ratio, thr)
        oa, ob, ta, tb, t = pyoracle.carryover(W, prob.astr, prob.bstr, L, kind, ratio, thr)
        np.testing.assert_array_equal(r["astr"], oa)
        np.testing.assert_array_equal(r["bstr"], ob)
        if ratio:
            assert r["truncated_a"] == pytest.approx(ta, abs=1e-12)
            assert r["truncated_b"] == pytest.approx(tb, abs=1e-12)
        if kind == 3:
            assert r["total_weight"] == pytest.approx(t, rel=1e-12)


@pytest.mark.gpu
def test_gpu_carryover_device_vector_capacity_and_davidson_hook():
    """Device-resident W gives the same strings; a short buffer returns SBD_TPB_ERR_CAPACITY with
    the counts; Davidson's carry-over of its own final vector equals the oracle's on that vector."""
    import ctypes as C
    import pyoracle
    import sbd_tpb
    import torch
    prob, g, meta = golden_problem("syn12_co")
    ratio, thr, cut, *_ = _ref_outputs(g)
    h = _handle(prob)
    dW = torch.from_numpy(g["W"]).cuda()
    r = h.carryover(dW, sbd_tpb.CARRYOVER_DOMINANT_SINGLES, 0.0, thr, mem=sbd_tpb.DEVICE)
    np.testing.assert_array_equal(r["astr"], g["co2_a"])
    co = sbd_tpb.Carryover(type=1, ratio=0.0, threshold=thr)
    buf = np.zeros(3, np.uint64)
    co.astr = buf.ctypes.data_as(C.POINTER(C.c_uint64))
    co.acap = 3
    w = np.ascontiguousarray(g["W"])
    rc = sbd_tpb.lib().sbd_tpb_carryover_strings(h.h, w.ctypes.data, sbd_tpb.HOST, C.byref(co))
    assert rc == sbd_tpb.ERR_CAPACITY
    assert co.na == len(g["co1_a"]) and co.nb == len(g["co1_b"])
    res = h.davidson(sbd_tpb.default_params(max_it=10, max_nb=10, eps=1e-10), want_vector=True,
                     carryover=(sbd_tpb.CARRYOVER_CUTOFF_SINGLES, 0.0, cut))
    # the library's W is in the reference convention; only W^2 enters
    oa, ob, _, _, t = pyoracle.carryover(res["W"], prob.astr, prob.bstr, prob.norb, 3, 0.0, cut)
    np.testing.assert_array_equal(res["carryover"]["astr"], oa)
    np.testing.assert_array_equal(res["carryover"]["bstr"], ob)
    assert res["carryover"]["total_weight"] == pytest.approx(t, rel=1e-12)


@pytest.mark.gpu
def test_cli_carryover_files(tmp_path):
    """--carryover_type 1 with --carryover_ratio prints the truncated weights and writes the string
    files; the strings equal the oracle's on the CLI's own saved vector."""
    import pyoracle
    import synth
    prob, g, meta = golden_problem("syn12_co")
    DIAG = os.path.join(ROOT, "sbd-pub_b200", "bin", "diag")
    fcidump, alpha, beta = (str(tmp_path / f) for f in ("fcidump.txt", "a.txt", "b.txt"))
    synth.write_fcidump(fcidump, prob.norb, prob.nelec, prob.h1, prob.eri_packed, prob.core)
    synth.write_strings(alpha, prob.astr, prob.norb)
    synth.write_strings(beta, prob.bstr, prob.norb)
    cmd = [DIAG, "--fcidump", fcidump, "--adetfile", alpha, "--bdetfile", beta, "--iteration", "10",
           "--block", "10", "--tolerance", "1e-10", "--carryover_type", "1", "--carryover_ratio", "0.25",
           "--carryover_adetfile", "co_a.txt", "--carryover_bdetfile", "co_b.txt", "--savename", "wf"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    from test_cli import read_wavefunction
    _, _, _, W = read_wavefunction(str(tmp_path / "wf000000"))
    oa, ob, ta, tb, _ = pyoracle.carryover(W, prob.astr, prob.bstr, prob.norb, 1, 0.25, 0.01)
    to_int = lambda f: [int(l.strip(), 2) for l in open(tmp_path / f) if l.strip()]  # noqa: E731
    assert to_int("co_a.txt") == [int(x) for x in oa]
    assert to_int("co_b.txt") == [int(x) for x in ob]
    m = re.search(r"truncated weight in carry-over for alpha-det = ([-0-9.eE+]+)", r.stdout)
    assert m and float(m.group(1)) == pytest.approx(ta, abs=1e-12)
    m = re.search(r"carryover bitstrings = \[(.*)\], size = (\d+)", r.stdout)
    assert m and int(m.group(2)) == len(oa)
