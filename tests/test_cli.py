"""The drop-in CLI (sbd-pub_b200/bin/diag) with the reference app's flags, run on FCIDUMP and
string files written from the n2 fixture: the energy line matches the reference's energy and the
RDM files and energy decomposition are produced (GPU)."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden_cases, golden_problem

DIAG = os.path.join(ROOT, "sbd-pub_b200", "bin", "diag")


def test_cli_binary_built_and_rejects_bad_flags(tmp_path):
    assert os.path.exists(DIAG), "build with make -C sbd-pub_b200"
    r = subprocess.run([DIAG, "--method", "3"], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0


@pytest.mark.gpu
def test_cli_n2_energy_and_rdm(tmp_path):
    import synth
    prob, g, meta = golden_problem("n2_1em3")
    fcidump = str(tmp_path / "fcidump.txt")
    alpha = str(tmp_path / "alpha.txt")
    synth.write_fcidump(fcidump, prob.norb, prob.nelec, prob.h1, prob.eri_packed, prob.core)
    synth.write_strings(alpha, prob.astr, prob.norb)
    it, nb, eps = meta["davidson"]
    cmd = [DIAG, "--fcidump", fcidump, "--adetfile", alpha, "--method", "0", "--iteration", str(it),
           "--block", str(nb), "--tolerance", str(eps), "--rdm", "1"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    m = re.search(r"^ Energy = ([-0-9.eE+]+)", r.stdout, re.M)
    assert m, r.stdout
    assert float(m.group(1)) == pytest.approx(golden_cases()["n2_1em3"]["energy"], abs=1e-8)
    tot = re.search(r"Zero-Body \+ One-Body \+ Two-Body energy = ([-0-9.eE+]+)", r.stdout)
    assert tot and float(tot.group(1)) == pytest.approx(float(m.group(1)), abs=1e-7)
    for f in ("1pRDM.txt", "2pRDM.txt"):
        assert os.path.getsize(tmp_path / f) > 0


def read_wavefunction(path):
    """The reference's one-rank wavefunction file (tpb/restart.h): counts, string words, W."""
    raw = open(path, "rb").read()
    na, nb, ln = np.frombuffer(raw[:24], np.uint64)
    na, nb, ln = int(na), int(nb), int(ln)
    words = np.frombuffer(raw[24:24 + 8 * ln * (na + nb)], np.uint64).reshape(na + nb, ln)
    W = np.frombuffer(raw[24 + 8 * ln * (na + nb):], np.float64)
    return na, nb, words, W


@pytest.mark.gpu
def test_cli_save_and_load_wavefunction(tmp_path):
    """--savename writes the reference's file layout; --loadname restarts from it and converges in
    the first step to the same energy."""
    import synth
    prob, g, meta = golden_problem("n2_1em3")
    fcidump = str(tmp_path / "fcidump.txt")
    alpha = str(tmp_path / "alpha.txt")
    synth.write_fcidump(fcidump, prob.norb, prob.nelec, prob.h1, prob.eri_packed, prob.core)
    synth.write_strings(alpha, prob.astr, prob.norb)
    base = [DIAG, "--fcidump", fcidump, "--adetfile", alpha, "--method", "0", "--iteration", "10",
            "--block", "10", "--tolerance", "1e-8", "--bit_length", "20"]
    r = subprocess.run(base + ["--savename", "wf"], capture_output=True, text=True, timeout=600,
                       cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    e1 = float(re.search(r"^ Energy = ([-0-9.eE+]+)", r.stdout, re.M).group(1))
    na, nb, words, W = read_wavefunction(str(tmp_path / "wf000000"))
    L = prob.norb
    assert (na, nb) == (len(prob.astr), len(prob.bstr)) and words.shape[1] == (L + 19) // 20
    # strings: bit p of the orbital string in word p // 20, bit p % 20
    for k, s in enumerate(list(prob.astr[:20])):
        v = sum(((int(words[k, p // 20]) >> (p % 20)) & 1) << p for p in range(L))
        assert v == int(s)
    assert abs(np.linalg.norm(W) - 1.0) < 1e-10
    r2 = subprocess.run(base + ["--loadname", "wf"], capture_output=True, text=True, timeout=600,
                        cwd=str(tmp_path))
    assert r2.returncode == 0, r2.stderr
    assert "Elapsed time for init" in r2.stdout
    e2 = float(re.search(r"^ Energy = ([-0-9.eE+]+)", r2.stdout, re.M).group(1))
    assert e2 == pytest.approx(e1, abs=1e-9)
    steps = re.findall(r"Davidson iteration \d+\.\d+", r2.stdout)
    assert len(steps) <= 2  # converged at once from the stored vector


def test_cli_missing_wavefunction_file(tmp_path):
    r = subprocess.run([DIAG, "--fcidump", str(tmp_path / "none.txt"), "--loadname", "nothing"],
                       capture_output=True, text=True, timeout=60, cwd=str(tmp_path))
    assert r.returncode != 0


@pytest.mark.gpu
def test_cli_learned_preconditioner_params(tmp_path):
    """--preconditioner learned with a parameter file: an untrained network (factor 1) gives the
    diagonal solver's energy; without a file the flag is rejected."""
    import sbd_tpb
    import synth
    prob, g, meta = golden_problem("n2_1em3")
    fcidump = str(tmp_path / "fcidump.txt")
    alpha = str(tmp_path / "alpha.txt")
    synth.write_fcidump(fcidump, prob.norb, prob.nelec, prob.h1, prob.eri_packed, prob.core)
    synth.write_strings(alpha, prob.astr, prob.norb)
    pc = sbd_tpb.Precond(0, seed=3)
    pc.get_params().tofile(str(tmp_path / "net.bin"))
    pc.close()
    base = [DIAG, "--fcidump", fcidump, "--adetfile", alpha, "--iteration", "10", "--block", "10",
            "--tolerance", "1e-8"]
    r = subprocess.run(base + ["--preconditioner", "learned", "--precond_params", "net.bin"],
                       capture_output=True, text=True, timeout=600, cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    e = float(re.search(r"^ Energy = ([-0-9.eE+]+)", r.stdout, re.M).group(1))
    assert e == pytest.approx(golden_cases()["n2_1em3"]["energy"], abs=1e-8)
    r2 = subprocess.run(base + ["--preconditioner", "learned"], capture_output=True, text=True, timeout=600,
                        cwd=str(tmp_path))
    assert r2.returncode != 0

