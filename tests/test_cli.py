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
