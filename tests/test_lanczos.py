"""Lanczos (--method 2; tpb/lanczos.h:167-320).

CPU: the oracle's restatement (orc_lanczos) against the reference's own sbd::Lanczos, run by
oracle/_ref/ref_dump --lanczos on the fixtures (tests/golden/make_golden.py): the same number of
step lines, the same final vector up to its global sign, the same energy <W|H|W>.  GPU: the
library's Lanczos (sbd_tpb_lanczos, sbd_tpb_diag with method 2, the CLI's --method 2) against
both.  Lanczos without reorthogonalisation amplifies rounding, and the reference restarts from and
reports <W|H|W> of an unnormalised W (the library renormalises it, which changes nothing on these
inputs), so energies are compared to 1e-7 relative (the fixtures' own spread between the oracle
and the reference is below 2e-8 relative).  The FCI-12 case shows why the library renormalises:
there the reference's restart vector drifts in norm and its iteration leaves the ground state."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden_cases, golden_problem

LZ_CASES = [n for n, m in golden_cases().items() if "lanczos" in m]


def _system(prob):
    import pyoracle
    ham = pyoracle.Hamiltonian.from_arrays(prob.norb, prob.nelec, prob.core, prob.h1, prob.eri_packed)
    return pyoracle.System(ham, prob.astr, prob.bstr)


def _same_up_to_sign(a, b):
    return min(np.abs(a - b).max(), np.abs(a + b).max())


@pytest.mark.parametrize("name", LZ_CASES)
def test_oracle_lanczos_matches_reference(name):
    prob, g, meta = golden_problem(name)
    it, nb, tol = meta["lanczos"]
    e_ref, lines_ref = float(g["lanczos"][0]), int(g["lanczos"][1])
    E, W, ns, printed, conv = _system(prob).lanczos(it, nb, tol)
    assert printed == lines_ref
    assert conv
    assert E == pytest.approx(e_ref, rel=1e-7)
    if "W_lanczos" in g:
        assert _same_up_to_sign(W, g["W_lanczos"]) < 1e-8


# ---------------------------------------------------------------------------------------------- GPU


@pytest.mark.gpu
@pytest.mark.parametrize("name", LZ_CASES)
def test_gpu_lanczos_matches_reference(name):
    import sbd_tpb
    prob, g, meta = golden_problem(name)
    it, nb, tol = meta["lanczos"]
    e_ref = float(g["lanczos"][0])
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    p = sbd_tpb.default_params(max_it=it, max_nb=nb, eps=tol, method=sbd_tpb.METHOD_LANCZOS)
    r = h.davidson(p, want_vector=True)
    E_or, W_or, ns_or, _, _ = _system(prob).lanczos(it, nb, tol)
    assert r["converged"]
    assert r["energy"] == pytest.approx(e_ref, rel=1e-7)
    assert abs(r["iterations"] - ns_or) <= 1
    if "W_lanczos" in g:
        assert _same_up_to_sign(r["W"], g["W_lanczos"]) < 1e-7
    assert _same_up_to_sign(r["W"], W_or) < 1e-7


@pytest.mark.gpu
def test_gpu_lanczos_reaches_davidson_energy_and_rejects_mixed():
    """With enough steps Lanczos reaches the Davidson ground state of n2 (the reference's own
    data set); the mixed-precision path is Davidson-only."""
    import sbd_tpb
    prob, g, meta = golden_problem("n2_1em3")
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    r = h.davidson(sbd_tpb.default_params(max_it=4, max_nb=60, eps=1e-10, method=sbd_tpb.METHOD_LANCZOS),
                   want_vector=True)
    assert r["energy"] == pytest.approx(float(g["energy"][0]), abs=1e-7)
    assert abs(np.linalg.norm(r["W"]) - 1.0) < 1e-6
    with pytest.raises(sbd_tpb.TpbError):
        h.davidson(sbd_tpb.default_params(method=sbd_tpb.METHOD_LANCZOS, precision=sbd_tpb.MIXED))


@pytest.mark.gpu
def test_cli_lanczos(tmp_path):
    """--method 2: the reference's " Lanczos iteration" lines, one per continued step, and the
    energy of the reference's Lanczos."""
    import synth
    prob, g, meta = golden_problem("syn8")
    it, nb, tol = meta["lanczos"]
    DIAG = os.path.join(ROOT, "sbd-pub_b200", "bin", "diag")
    fcidump, alpha = str(tmp_path / "fcidump.txt"), str(tmp_path / "a.txt")
    synth.write_fcidump(fcidump, prob.norb, prob.nelec, prob.h1, prob.eri_packed, prob.core)
    synth.write_strings(alpha, prob.astr, prob.norb)
    cmd = [DIAG, "--fcidump", fcidump, "--adetfile", alpha, "--method", "2", "--iteration", str(it),
           "--block", str(nb), "--tolerance", repr(tol)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith(" Lanczos iteration")]
    assert abs(len(lines) - int(g["lanczos"][1])) <= 1
    m = re.search(r"^ Energy = ([-0-9.eE+]+)", r.stdout, re.M)
    assert m and float(m.group(1)) == pytest.approx(float(g["lanczos"][0]), rel=1e-7)


@pytest.mark.gpu
def test_gpu_lanczos_fci12_stays_on_the_ground_state():
    """The 12-orbital FCI (853,776 determinants) to tolerance 1e-8 over 20 restarts: with the
    renormalised restart the energy reaches the reference's Davidson answer."""
    import sbd_tpb
    prob, g, meta = golden_problem("fci12")
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    r = h.davidson(sbd_tpb.default_params(max_it=20, max_nb=10, eps=1e-8, method=sbd_tpb.METHOD_LANCZOS),
                   want_vector=False)
    assert r["converged"]
    assert r["energy"] == pytest.approx(float(g["energy"][0]), abs=1e-7)
