"""String files (LoadAlphaDets, basic/makedeterminants.h:160-186): text and binary parsing, sort and
de-duplication on the GPU (sbd_tpb_parse_strings / sbd_tpb_read_strings, the CLI's readers).

CPU: the oracle's readers (orc_load_strings, orc_load_strings_bin) against what the reference's
own LoadAlphaDets made of the fixture files (tests/golden/strings.npz: unsorted text and binary
files with duplicates, CRLF line ends and random bits in the unused high bits of the binary
records).  GPU: the library against both, bit for bit, plus the edge cases and errors of the text
format and a few million strings."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, golden_cases

SIZES = [12, 20, 36]


def _fixture():
    return np.load(os.path.join(GOLDEN, "strings.npz"))


def _write(path, data):
    with open(path, "wb") as f:
        f.write(bytes(data))
    return str(path)


@pytest.mark.parametrize("L", SIZES)
def test_oracle_readers_match_reference(L, tmp_path):
    import pyoracle
    g = _fixture()
    t = _write(tmp_path / "a.txt", g[f"L{L}_txt_bytes"])
    b = _write(tmp_path / "a.bin", g[f"L{L}_bin_bytes"])
    np.testing.assert_array_equal(pyoracle.load_strings(t, L), g[f"L{L}_txt_ref"])
    np.testing.assert_array_equal(pyoracle.load_strings_bin(b, L), g[f"L{L}_bin_ref"])
    assert len(g[f"L{L}_txt_ref"]) == golden_cases()["strings"][f"L{L}"]["unique"]


# ---------------------------------------------------------------------------------------------- GPU


def _handle():
    import sbd_tpb
    return sbd_tpb.Handle(0)


@pytest.mark.gpu
@pytest.mark.parametrize("L", SIZES)
def test_gpu_strings_match_reference(L, tmp_path):
    import sbd_tpb
    g = _fixture()
    h = _handle()
    np.testing.assert_array_equal(h.parse_strings(g[f"L{L}_txt_bytes"], L), g[f"L{L}_txt_ref"])
    np.testing.assert_array_equal(h.parse_strings(g[f"L{L}_bin_bytes"], L, sbd_tpb.STRINGS_BINARY),
                                  g[f"L{L}_bin_ref"])
    t = _write(tmp_path / "a.txt", g[f"L{L}_txt_bytes"])
    b = _write(tmp_path / "a.bin", g[f"L{L}_bin_bytes"])
    np.testing.assert_array_equal(h.read_strings(t, L), g[f"L{L}_txt_ref"])
    np.testing.assert_array_equal(h.read_strings(b, L), g[f"L{L}_bin_ref"])


@pytest.mark.gpu
def test_gpu_text_edge_cases_against_oracle(tmp_path):
    """Trailing spaces and CR, blank lines, no final newline, characters after the first norb,
    widths 1 and 64, a binary file with a trailing partial record."""
    import pyoracle
    import sbd_tpb
    h = _handle()
    cases = {
        6: "000111  \r\n\n\n111000extra\n010101\r\n000111\n101010",
        1: "1\n0\n1\n\n",
        64: "\n".join(format(v, "064b") for v in (2**64 - 1, 1, 2**63, 12345678901234567)) + "\n",
    }
    for L, text in cases.items():
        p = _write(tmp_path / f"e{L}.txt", text.encode())
        np.testing.assert_array_equal(h.read_strings(p, L), pyoracle.load_strings(p, L))
    rng = np.random.default_rng(3)
    vals = rng.integers(0, 2**63, size=1000, dtype=np.uint64) * 2 + 1
    raw = b"".join(int(v).to_bytes(8, "big") for v in vals) + b"\x01\x02\x03"  # partial record
    p = _write(tmp_path / "w.bin", raw)
    out = h.read_strings(p, 64)
    np.testing.assert_array_equal(out, pyoracle.load_strings_bin(p, 64))
    np.testing.assert_array_equal(out, np.unique(vals))
    assert len(h.parse_strings(b"", 8)) == 0


@pytest.mark.gpu
def test_gpu_text_errors():
    import sbd_tpb
    h = _handle()
    with pytest.raises(sbd_tpb.TpbError, match="line 3 is shorter than norb"):
        h.parse_strings(b"0011\n0101\n011\n0110\n", 4)
    with pytest.raises(sbd_tpb.TpbError, match="line 2 has characters other than 0/1"):
        h.parse_strings(b"0011\n01x1\n0110\n01y0\n", 4)
    # the first failing line is reported whichever warp sees it first
    bad = b"".join(b"0011\n" for _ in range(5000)) + b"012\n" + b"0011\n" * 5000 + b"0x01\n"
    with pytest.raises(sbd_tpb.TpbError, match="line 5001 is shorter than norb"):
        h.parse_strings(bad, 4)
    # a buffer too small: the count comes back with SBD_TPB_ERR_CAPACITY
    import ctypes as C
    n = C.c_size_t(0)
    rc = sbd_tpb.lib().sbd_tpb_parse_strings(h.h, b"0011\n0101\n", 10, sbd_tpb.STRINGS_TEXT, 4, None, 0,
                                             C.byref(n))
    assert rc == sbd_tpb.ERR_CAPACITY and n.value == 2


@pytest.mark.gpu
@pytest.mark.parametrize("fmt", ["txt", "bin"])
def test_gpu_strings_at_size(fmt, tmp_path):
    """Two million 40-orbital strings with duplicates, unsorted: equal to the oracle's reader."""
    import pyoracle
    rng = np.random.default_rng(11)
    L = 40
    vals = rng.integers(0, 2**L, size=2_000_000, dtype=np.uint64)
    vals = np.concatenate([vals, vals[:300_000]])
    rng.shuffle(vals)
    if fmt == "txt":
        bits = ((vals[:, None] >> np.arange(L - 1, -1, -1, dtype=np.uint64)) & 1).astype(np.uint8)
        lines = np.concatenate([bits + ord("0"), np.full((len(vals), 1), ord("\n"), np.uint8)], axis=1)
        p = _write(tmp_path / "big.txt", lines.tobytes())
        ref = pyoracle.load_strings(p, L)
    else:
        recs = (vals[:, None] >> np.arange(32, -1, -8, dtype=np.uint64)[None, :] & 0xFF).astype(np.uint8)
        p = _write(tmp_path / "big.bin", recs.tobytes())
        ref = pyoracle.load_strings_bin(p, L)
    h = _handle()
    out = h.read_strings(p, L)
    np.testing.assert_array_equal(out, ref)
    np.testing.assert_array_equal(out, np.unique(vals))


@pytest.mark.gpu
def test_cli_reads_binary_string_files(tmp_path):
    """The CLI takes a .bin string file (rejected before this reader existed) and gives the same
    energy as the text form of the same strings."""
    import re
    import subprocess

    import synth
    from conftest import golden_problem
    prob, g, meta = golden_problem("syn8")
    DIAG = os.path.join(ROOT, "sbd-pub_b200", "bin", "diag")
    fd = str(tmp_path / "fcidump.txt")
    synth.write_fcidump(fd, prob.norb, prob.nelec, prob.h1, prob.eri_packed, prob.core)
    synth.write_strings(str(tmp_path / "a.txt"), prob.astr, prob.norb)
    rb = (prob.norb + 7) // 8
    _write(tmp_path / "a.bin", b"".join(int(s).to_bytes(rb, "big") for s in prob.astr[::-1]))
    energies = []
    for f in ("a.txt", "a.bin"):
        r = subprocess.run([DIAG, "--fcidump", fd, "--adetfile", str(tmp_path / f), "--iteration", "10",
                            "--block", "10", "--tolerance", "1e-10"], capture_output=True, text=True,
                           timeout=600, cwd=str(tmp_path))
        assert r.returncode == 0, r.stderr
        energies.append(float(re.search(r"^ Energy = ([-0-9.eE+]+)", r.stdout, re.M).group(1)))
    assert energies[0] == pytest.approx(float(g["energy"][0]), abs=1e-9)
    assert energies[1] == energies[0]
