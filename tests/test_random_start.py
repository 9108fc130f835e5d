"""The reference's seeded random start: --init 1 --seed S (BasisInitVector with init 1,
tpb/davidson.h:138-141; Randomize, framework/dm_vector.h:100-178).

CPU: the oracle's restatement of the generator reproduces the start vector the reference wrote
(ref_dump --init 1 SEED, w0.f64: every entry of syn8, sampled entries and checksums of n2 1e-3),
and the oracle's Davidson from that start reaches the reference's energy.
GPU: the library's Davidson from --init 1 (FP64 and mixed precision) reaches the reference's
energy, its vector equals the reference's up to sign (syn8), the drop-in CLI takes --init 1 --seed,
and symmetry 2 (the random start projected onto the exchange-symmetric sector) reaches the same
state as the unprojected start on a problem whose lowest state is exchange-symmetric."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden_problem

CASES = ["syn8_init1", "n2_1em3_init1"]


def _w0(name):
    prob, g, meta = golden_problem(name)
    return prob, g, meta, int(meta["init"][1])


@pytest.mark.parametrize("name", CASES)
def test_oracle_random_start_matches_reference(name):
    import pyoracle
    prob, g, meta, seed = _w0(name)
    n = len(prob.astr) * len(prob.bstr)
    w = pyoracle.random_start(n, seed)
    if "w0" in g:
        # the reference normalises with per-thread Kahan sums: the last bit can differ
        assert np.abs(w - g["w0"]).max() < 1e-15
    np.testing.assert_allclose(w[g["idx"]], g["w0_sample"], rtol=0, atol=1e-15)
    s = g["w0_sum"]
    assert abs(w.sum() - s[0]) < 1e-12 and abs((w * w).sum() - s[1]) < 1e-12
    # the unnormalised values are the hash bits exactly: uniform in [-1, 1) on the 2^-52 grid
    raw = pyoracle.random_start(64, seed, normalise=False)
    assert np.all(np.abs(raw) <= 1.0) and np.array_equal(raw, np.round(raw * 2.0 ** 52) / 2.0 ** 52)


def test_oracle_davidson_from_random_start():
    import pyoracle
    prob, g, meta, seed = _w0("syn8_init1")
    ham = pyoracle.Hamiltonian.from_arrays(prob.norb, prob.nelec, prob.core, prob.h1, prob.eri_packed)
    sysm = pyoracle.System(ham, prob.astr, prob.bstr)
    it, nb, tol = meta["davidson"]
    e, W, _, _ = sysm.davidson(max_it=it, max_nb=nb, eps=tol, W0=pyoracle.random_start(sysm.na * sysm.nb, seed))
    assert e == pytest.approx(meta["energy"], abs=1e-10)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_gpu_davidson_random_start(name, prec):
    import sbd_tpb
    prob, g, meta, seed = _w0(name)
    it, nb, tol = meta["davidson"]
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    fp64 = prec == "fp64"
    r = h.davidson(sbd_tpb.default_params(max_it=it, max_nb=nb, eps=tol if fp64 else 1e-5, init=1, seed=seed,
                                          precision=sbd_tpb.FP64 if fp64 else sbd_tpb.MIXED), want_vector=True)
    h.close()
    assert r["converged"]
    assert r["energy"] == pytest.approx(meta["energy"], abs=1e-8 if fp64 else 1e-6)
    if fp64 and "W" in g:
        W = r["W"]
        assert min(np.abs(W - g["W"]).max(), np.abs(W + g["W"]).max()) < 1e-6


@pytest.mark.gpu
def test_gpu_random_start_seed_and_projection():
    """Different seeds, the same lowest state; symmetry 2 (projected random start) reaches it too
    (syn8: alpha and beta lists identical)."""
    import sbd_tpb
    prob, g, meta, seed = _w0("syn8_init1")
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    es = []
    for s_, sym in ((seed, 0), (seed + 1, 0), (seed, 2)):
        r = h.davidson(sbd_tpb.default_params(max_it=30, max_nb=10, eps=1e-10, init=1, seed=s_, symmetry=sym),
                       want_vector=False)
        assert r["converged"]
        es.append(r["energy"])
    h.close()
    assert max(es) - min(es) < 1e-9 and abs(es[0] - meta["energy"]) < 1e-9


@pytest.mark.gpu
def test_gpu_invalid_init_rejected():
    import sbd_tpb
    prob, g, meta, seed = _w0("syn8_init1")
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    with pytest.raises(RuntimeError, match="init must be 0 or 1"):
        h.davidson(sbd_tpb.default_params(init=2), want_vector=False)
    h.close()


@pytest.mark.gpu
def test_gpu_cli_random_start(tmp_path):
    import synth
    prob, g, meta, seed = _w0("n2_1em3_init1")
    fcidump, alpha = str(tmp_path / "fcidump.txt"), str(tmp_path / "alpha.txt")
    synth.write_fcidump(fcidump, prob.norb, prob.nelec, prob.h1, prob.eri_packed, prob.core)
    synth.write_strings(alpha, prob.astr, prob.norb)
    it, nb, tol = meta["davidson"]
    out = subprocess.run([os.path.join(ROOT, "sbd-pub_b200", "bin", "diag"), "--fcidump", fcidump, "--adetfile",
                          alpha, "--iteration", str(it), "--block", str(nb), "--tolerance", repr(tol),
                          "--init", "1", "--seed", str(seed)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    e = float(re.search(r"Sample-based diagonalization: Energy = ([-0-9.eE+]+)", out.stdout).group(1))
    assert e == pytest.approx(meta["energy"], abs=1e-8)
