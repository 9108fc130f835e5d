"""The drop-in CLI (sbd-pub_b200/bin/diag) with the reference app's flags, run on FCIDUMP and
string files written from the n2 fixture: the energy line matches the reference's energy and the
RDM files and energy decomposition are produced (GPU).  On the CPU: its flag checks, FCIDUMP errors
and the error it stops with when there is no device."""
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


# Host-side checks that run before any device call: flag values the drop-in does not build (the
# reference app accepts them, main.cc) and malformed FCIDUMP files (fcidump.h:29-141 reads them)
BAD_FLAGS = [
    (["--method", "1"], "only the matrix-free solvers are built"),
    (["--method", "3"], "only the matrix-free solvers are built"),
    (["--bit_length", "0"], "--bit_length must be in [1, 64]"),
    (["--bit_length", "65"], "--bit_length must be in [1, 64]"),
    (["--adet_comm_size", "2"], "one rank on one GPU: --*_comm_size must be 1"),
    (["--task_comm_size", "4"], "one rank on one GPU: --*_comm_size must be 1"),
    (["--init", "2"], "--init must be 0 (first determinant) or 1 (seeded random vector)"),
    (["--carryover_type", "4"], "--carryover_type must be 0, 1, 2 or 3"),
    (["--precision", "fp16"], "--precision must be fp64 or mixed"),
    (["--preconditioner", "jacobi"], "--preconditioner must be diagonal or learned"),
    (["--dump_matrix_form_wf", "wf.txt"], "not built in this version: --dump_matrix_form_wf"),
    (["--tolerance"], "missing value for --tolerance"),
]


@pytest.mark.parametrize("args,msg", BAD_FLAGS)
def test_cli_flag_errors(args, msg, tmp_path):
    r = subprocess.run([DIAG] + args, capture_output=True, text=True, timeout=60, cwd=str(tmp_path))
    assert r.returncode == 1
    assert r.stderr.startswith("diag: ") and msg in r.stderr


FCIDUMPS = {
    "no_norb": (" &FCI NELEC=2,MS2=0,\n &END\n 0.5 1 1 1 1\n", "FCIDUMP header has no NORB"),
    "norb_65": (" &FCI NORB=65,NELEC=2,\n &END\n 0.5 1 1 1 1\n", "NORB must be in [1, 64]"),
    "one_body_index": (" &FCI NORB=2,NELEC=2,\n &END\n -1.0 3 1 0 0\n", "one-electron index out of range"),
    "two_body_index": (" &FCI NORB=2,NELEC=2,\n &END\n 0.5 1 1 2 3\n", "two-electron index out of range"),
}


@pytest.mark.parametrize("case", sorted(FCIDUMPS))
def test_cli_fcidump_errors(case, tmp_path):
    text, msg = FCIDUMPS[case]
    (tmp_path / "fcidump.txt").write_text(text)
    r = subprocess.run([DIAG, "--fcidump", str(tmp_path / "fcidump.txt")], capture_output=True, text=True,
                       timeout=60, cwd=str(tmp_path))
    assert r.returncode == 1 and msg in r.stderr
    r = subprocess.run([DIAG, "--fcidump", str(tmp_path / "missing.txt")], capture_output=True, text=True,
                       timeout=60, cwd=str(tmp_path))
    assert r.returncode == 1 and "Failed to open FCIDUMP file" in r.stderr


def test_cli_fails_loudly_without_a_device(tmp_path):
    """A valid input on a machine without a GPU: the CLI stops with the library's error (there is
    no CPU fallback)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    (tmp_path / "fcidump.txt").write_text(" &FCI NORB=2,NELEC=2,MS2=0,\n &END\n 0.5 1 1 1 1\n -1.0 1 1 0 0\n"
                                          " -0.5 2 2 0 0\n 0.1 0 0 0 0\n")
    (tmp_path / "a.txt").write_text("01\n10\n")
    r = subprocess.run([DIAG, "--fcidump", "fcidump.txt", "--adetfile", "a.txt"], capture_output=True, text=True,
                       timeout=60, cwd=str(tmp_path))
    assert r.returncode == 1 and r.stderr.strip() == "diag: no CUDA device"


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

