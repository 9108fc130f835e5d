"""The oracle's sigma against the dense Hamiltonian built from its own element function
(orc_hij, the reference's Hij on interleaved determinants) on the edge shapes the GPU edge tests
use: shuffled strings, one determinant, strings without connections, 64-orbital strings."""
import numpy as np
import pytest

from test_gpu_edges import _problem, _random_strings


def _dense_check(prob):
    import pyoracle
    ham = pyoracle.Hamiltonian.from_arrays(prob.norb, prob.nelec, prob.core, prob.h1, prob.eri_packed)
    s = pyoracle.System(ham, prob.astr, prob.bstr)
    na, nb = len(prob.astr), len(prob.bstr)
    H = np.zeros((na * nb, na * nb))
    for i in range(na * nb):
        for j in range(na * nb):
            H[i, j] = s.hij(prob.astr[i // nb], prob.bstr[i % nb], prob.astr[j // nb], prob.bstr[j % nb])
    x = np.random.default_rng(0).normal(size=na * nb)
    ref = H @ x
    assert np.max(np.abs(s.sigma(x) - ref)) <= 1e-13 * max(np.max(np.abs(ref)), 1.0)
    np.testing.assert_allclose(s.diagonal(), np.diag(H), rtol=1e-14, atol=1e-12)


def test_oracle_dense_shuffled():
    rng = np.random.default_rng(9)
    a = _random_strings(10, 4, 12, rng)
    b = _random_strings(10, 4, 11, rng)
    pa, pb = rng.permutation(len(a)), rng.permutation(len(b))
    _dense_check(_problem(10, 4, 4, [a[i] for i in pa], [b[i] for i in pb]))


@pytest.mark.parametrize("strings", [[0b11], [0b000111, 0b111000]])
def test_oracle_dense_degenerate(strings):
    n = bin(strings[0]).count("1")
    _dense_check(_problem(6, n, n, strings, strings))


def test_oracle_dense_64_orbitals():
    rng = np.random.default_rng(5)
    a = sorted(set([(1 << 3) - 1] + _random_strings(64, 3, 8, rng)))
    b = sorted(set([(1 << 3) - 1] + _random_strings(64, 3, 7, rng)))
    _dense_check(_problem(64, 3, 3, a, b))
