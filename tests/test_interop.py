"""Interoperability with the reference itself (needs a B200 and oracle/_ref built from the
reference's sources).

* Wavefunction files in both directions: the reference app's --savename file (SaveWavefunction,
  tpb/restart.h:21-66, called at tpb/sbdiag.h:743) read by the drop-in CLI's --loadname, and the
  CLI's --savename file read by the reference app's --loadname (LoadWavefunction, tpb/restart.h:415,
  called at tpb/sbdiag.h:288): energies and W agree.
* The drop-in binding include/sbd_tpb_sbd.hpp, compiled against the reference's headers
  (oracle/_ref/binding_check), run through the app's flow beside the reference's own
  sbd::tpb::diag (tpb/sbdiag.h:139-151): energy, occupations, RDMs and carry-over strings agree.

Inputs are the n2 fixture's FCIDUMP and strings (data/n2 of the reference), written to files.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden_problem
from test_cli import read_wavefunction

pytestmark = pytest.mark.gpu

DIAG = os.path.join(ROOT, "sbd-pub_b200", "bin", "diag")
REF_DIAG = os.path.join(ROOT, "oracle", "_ref", "diag")
BINDING = os.path.join(ROOT, "oracle", "_ref", "binding_check")
needs_ref = pytest.mark.skipif(not (os.path.exists(REF_DIAG) and os.path.exists(BINDING)),
                               reason="oracle/_ref not built (needs the reference checkout at build time)")


def _inputs(tmp_path):
    import synth
    prob, g, meta = golden_problem("n2_1em3")
    fcidump, alpha = str(tmp_path / "fcidump.txt"), str(tmp_path / "alpha.txt")
    synth.write_fcidump(fcidump, prob.norb, prob.nelec, prob.h1, prob.eri_packed, prob.core)
    synth.write_strings(alpha, prob.astr, prob.norb)
    return prob, meta, ["--fcidump", fcidump, "--adetfile", alpha, "--method", "0"]


def _energy(out):
    return float(re.search(r"Sample-based diagonalization: Energy = ([-0-9.eE+]+)", out).group(1))


def _run(cmd, cwd, threads=None):
    env = dict(os.environ, OMP_NUM_THREADS=str(threads or os.cpu_count()))
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=900, cwd=str(cwd), env=env)
    assert r.returncode == 0, (cmd, r.stderr[-2000:])
    return r.stdout


def _same_up_to_sign(a, b):
    return min(np.abs(a - b).max(), np.abs(a + b).max())


@needs_ref
def test_reference_file_read_by_library(tmp_path):
    prob, meta, base = _inputs(tmp_path)
    solve = ["--iteration", "10", "--block", "10", "--tolerance", "1e-8"]
    ref_out = _run([REF_DIAG] + base + solve + ["--savename", "ref_"], tmp_path)
    e_ref = _energy(ref_out)
    assert e_ref == pytest.approx(meta["energy"], abs=1e-8)
    na, nb, words, W_ref = read_wavefunction(str(tmp_path / "ref_000000"))
    assert (na, nb) == (len(prob.astr), len(prob.bstr))
    # the library restarts from the reference's converged vector: one step, same energy, and the
    # vector it saves is the reference's
    out = _run([DIAG] + base + solve + ["--loadname", "ref_", "--savename", "lib_"], tmp_path)
    assert _energy(out) == pytest.approx(e_ref, abs=1e-8)
    assert len(re.findall(r"Davidson iteration \d+\.\d+", out)) <= 2
    na2, nb2, words2, W_lib = read_wavefunction(str(tmp_path / "lib_000000"))
    assert (na2, nb2) == (na, nb) and np.array_equal(words, words2)
    assert _same_up_to_sign(W_lib, W_ref) < 1e-9


@needs_ref
def test_library_file_read_by_reference(tmp_path):
    prob, meta, base = _inputs(tmp_path)
    out = _run([DIAG] + base + ["--iteration", "10", "--block", "10", "--tolerance", "1e-8",
                                "--savename", "lib_"], tmp_path)
    e_lib = _energy(out)
    assert e_lib == pytest.approx(meta["energy"], abs=1e-8)
    # the reference restarts from the library's vector: its first residual is already below the
    # tolerance and it saves the vector it read, normalised
    ref_out = _run([REF_DIAG] + base + ["--iteration", "2", "--block", "2", "--tolerance", "1e-7",
                                        "--loadname", "lib_", "--savename", "ref_"], tmp_path)
    assert _energy(ref_out) == pytest.approx(e_lib, abs=1e-8)
    tols = [float(x) for x in re.findall(r"Davidson iteration \d+\.\d+ \(tol=([-0-9.eE+]+)\)", ref_out)]
    assert tols and tols[0] < 1e-7
    _, _, words_l, W_lib = read_wavefunction(str(tmp_path / "lib_000000"))
    _, _, words_r, W_ref = read_wavefunction(str(tmp_path / "ref_000000"))
    assert np.array_equal(words_l, words_r)
    assert _same_up_to_sign(W_lib, W_ref) < 1e-9


@needs_ref
def test_binding_matches_reference_diag(tmp_path):
    prob, meta, base = _inputs(tmp_path)
    out = _run([BINDING] + base[:4] + ["--iteration", "10", "--block", "10", "--tolerance", "1e-8", "--rdm",
                                      "--carryover_type", "1", "--carryover_threshold", "0.01"], tmp_path)
    kv = dict(tok.split("=", 1) for tok in out.strip().splitlines()[-1].split())
    assert abs(float(kv["e_ref"]) - float(kv["e_b200"])) < 1e-8, kv
    assert abs(float(kv["e_b200"]) - meta["energy"]) < 1e-8, kv
    assert float(kv["density_diff"]) < 1e-6, kv
    assert float(kv["rdm1_diff"]) < 1e-6 and float(kv["rdm2_diff"]) < 1e-6, kv
    # the same carry-over strings (as sets: strings of equal weight may be ordered differently by
    # rounding-level differences of the two vectors, and the next load sorts them)
    assert kv["co_equal"] == "1" and int(kv["co_a"]) > 0, kv
    print(f"\nbinding vs sbd::tpb::diag: dE {abs(float(kv['e_ref']) - float(kv['e_b200'])):.1e}, carry-over "
          f"{kv['co_a']}/{kv['co_b']} strings, same order: {kv['co_same_order']}")


@needs_ref
def test_binding_restart_files(tmp_path):
    """The binding's --savename / --loadname go through the reference's own restart functions."""
    prob, meta, base = _inputs(tmp_path)
    args = base[:4] + ["--iteration", "10", "--block", "10", "--tolerance", "1e-8"]
    out = _run([BINDING] + args + ["--savename", "b_", "--skip_reference"], tmp_path)
    e1 = float(dict(tok.split("=", 1) for tok in out.strip().splitlines()[-1].split())["e_b200"])
    out2 = _run([BINDING] + args + ["--loadname", "b_"], tmp_path)
    kv = dict(tok.split("=", 1) for tok in out2.strip().splitlines()[-1].split())
    assert abs(float(kv["e_b200"]) - e1) < 1e-9 and abs(float(kv["e_ref"]) - e1) < 1e-8, kv


@needs_ref
def test_binding_random_start_matches_reference(tmp_path):
    """--init 1 --seed: the reference's sbd::tpb::diag and the binding start from the same seeded random
    vector (BasisInitVector with init 1, tpb/davidson.h:138-141) and reach the same energy and RDMs."""
    prob, meta, base = _inputs(tmp_path)
    out = _run([BINDING] + base[:4] + ["--iteration", "30", "--block", "10", "--tolerance", "1e-8", "--rdm",
                                      "--init", "1", "--seed", "4242"], tmp_path)
    kv = dict(tok.split("=", 1) for tok in out.strip().splitlines()[-1].split())
    assert abs(float(kv["e_ref"]) - float(kv["e_b200"])) < 1e-8, kv
    assert abs(float(kv["e_b200"]) - meta["energy"]) < 1e-8, kv
    assert float(kv["rdm1_diff"]) < 1e-6 and float(kv["rdm2_diff"]) < 1e-6, kv
