"""Synthetic-input generator and FCIDUMP / string I/O (host logic, CPU only)."""
import math

import numpy as np

import synth


def test_hamiltonian_symmetry_and_determinism():
    h1, eri, core = synth.synthetic_hamiltonian(10)
    h1b, erib, _ = synth.synthetic_hamiltonian(10)
    assert np.array_equal(h1, h1b) and np.array_equal(eri, erib) and core == 0.0
    assert np.allclose(h1, h1.T)
    assert np.allclose(np.diag(h1), -2 + 4 * np.arange(10) / 10)
    E = synth.unpack_eri(eri, 10)
    assert np.allclose(E, E.transpose(1, 0, 2, 3)) and np.allclose(E, E.transpose(2, 3, 0, 1))
    assert (np.einsum("ppqq->pq", E) > 0).all()
    assert np.array_equal(synth.pack_eri(E), eri)


def test_string_sampler():
    L, n = 20, 6
    s = synth.sample_strings(L, n, 500)
    assert len(s) == 500 and len(np.unique(s)) == 500
    assert np.all(np.diff(s.astype(np.int64)) > 0)
    assert int(s[0]) == (1 << n) - 1  # HF is the smallest string
    assert all(bin(int(x)).count("1") == n for x in s)
    assert np.array_equal(s, synth.sample_strings(L, n, 500))
    full = synth.sample_strings(8, 3, 10 ** 6)
    assert len(full) == math.comb(8, 3)


def test_fcidump_roundtrip(tmp_path, oracle):
    L = 7
    h1, eri, core = synth.synthetic_hamiltonian(L, seed=3)
    p = str(tmp_path / "fd.txt")
    synth.write_fcidump(p, L, 6, h1, eri, core + 1.25)
    L2, ne, h1b, erib, coreb = synth.read_fcidump(p)
    assert (L2, ne, coreb) == (L, 6, core + 1.25)
    assert np.array_equal(h1, h1b) and np.array_equal(eri, erib)
    # the oracle's restatement of framework/fcidump.h reads the same values
    ham = oracle.Hamiltonian.from_fcidump(p)
    assert np.array_equal(ham.h1(), h1) and np.array_equal(ham.eri_packed(), eri) and ham.I0 == core + 1.25


def test_string_file_roundtrip(tmp_path, oracle):
    s = synth.sample_strings(16, 5, 300)
    p = str(tmp_path / "a.txt")
    synth.write_strings(p, s[::-1], 16)  # unsorted on disk; readers sort and dedupe
    assert np.array_equal(synth.read_strings(p, 16), s)
    assert np.array_equal(oracle.load_strings(p, 16), s)
