"""Edge cases of the GPU path against the CPU oracle (needs a B200): one determinant, strings
without any connection, the widest strings (64 orbitals), row lengths that are not a multiple of
the 16-byte column groups (FP64 and FP32 scalar tails), shuffled string order, different alpha and
beta electron counts, the largest Davidson subspace and the smallest one with many restarts.
The oracle itself is checked on these shapes against the dense Hamiltonian built from its element
function in test_oracle_dense.py."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(L, na_el, nb_el, astr, bstr, seed=1729):
    import synth
    from sbd_tpb import Problem
    h1, eri, core = synth.synthetic_hamiltonian(L, seed=seed)
    return Problem(norb=L, nelec=na_el + nb_el, core=core, h1=h1, eri_packed=eri,
                   astr=np.asarray(astr, np.uint64), bstr=np.asarray(bstr, np.uint64))


def _check_sigma(prob, tol64=1e-12, tol32=2e-6):
    import pyoracle
    import sbd_tpb
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    ham = pyoracle.Hamiltonian.from_arrays(prob.norb, prob.nelec, prob.core, prob.h1, prob.eri_packed)
    s = pyoracle.System(ham, prob.astr, prob.bstr)
    x = np.random.default_rng(11).normal(size=prob.ndet)
    ref = s.sigma(x)
    scale = max(np.max(np.abs(ref)), 1e-300)
    out = h.sigma(x)
    assert np.max(np.abs(out - ref)) <= tol64 * scale
    out32 = h.sigma(x.astype(np.float32))
    assert np.max(np.abs(out32 - ref)) <= tol32 * scale
    hii = h.diagonal()
    np.testing.assert_allclose(hii, s.diagonal(), rtol=1e-13, atol=1e-11)
    return h, s


def _random_strings(L, n, count, rng):
    out = set()
    while len(out) < count:
        out.add(sum(1 << int(p) for p in rng.choice(L, n, replace=False)))
    return sorted(out)


def test_single_determinant():
    """One alpha and one beta string: sigma = H_00 C and Davidson returns H_00 at once."""
    import sbd_tpb
    prob = _problem(6, 2, 2, [0b11], [0b11])
    h, s = _check_sigma(prob)
    r = h.davidson(sbd_tpb.default_params(max_it=2, max_nb=4, eps=1e-10), want_vector=True)
    assert r["energy"] == pytest.approx(float(h.diagonal()[0]), abs=1e-12)
    assert abs(abs(r["W"][0]) - 1.0) < 1e-12


def test_strings_without_connections():
    """Strings three or more excitations apart: no singles or doubles anywhere, sigma = H_ii C."""
    import sbd_tpb
    a = [0b000111, 0b111000]
    prob = _problem(6, 3, 3, a, a)
    h, s = _check_sigma(prob)
    for kind in range(4):
        off, ket, cran = h.table(kind)
        assert ket.size == 0 and np.all(off == 0)
    x = np.random.default_rng(2).normal(size=prob.ndet)
    np.testing.assert_allclose(h.sigma(x), h.diagonal() * x, rtol=1e-14)


def test_widest_strings_64_orbitals():
    """norb = 64: every bit of the uint64 strings is an orbital."""
    rng = np.random.default_rng(5)
    L = 64
    a = sorted(set([(1 << 3) - 1] + _random_strings(L, 3, 40, rng)))
    b = sorted(set([(1 << 3) - 1] + _random_strings(L, 3, 33, rng)))
    prob = _problem(L, 3, 3, a, b)
    _check_sigma(prob)


@pytest.mark.parametrize("na,nb", [(37, 29), (61, 45), (130, 7)])
def test_ragged_sizes(na, nb):
    """Row lengths not a multiple of 4 (FP32) or 2 (FP64): the scalar tails of the block kernel
    and of every vector pass, and a last slab narrower than the rest."""
    import sbd_tpb
    rng = np.random.default_rng(na * 100 + nb)
    L = 12
    a = sorted(set([(1 << 4) - 1] + _random_strings(L, 4, na - 1, rng)))[:na]
    b = sorted(set([(1 << 3) - 1] + _random_strings(L, 3, nb - 1, rng)))[:nb]
    prob = _problem(L, 4, 3, a, b)
    h, s = _check_sigma(prob)
    e_or = s.davidson(max_it=20, max_nb=8, eps=1e-9)[0]
    r = h.davidson(sbd_tpb.default_params(max_it=20, max_nb=8, eps=1e-9), want_vector=False)
    assert r["energy"] == pytest.approx(e_or, abs=1e-8)
    rm = h.davidson(sbd_tpb.default_params(max_it=40, max_nb=8, eps=1e-5, precision=sbd_tpb.MIXED),
                    want_vector=False)
    assert rm["energy"] == pytest.approx(e_or, abs=1e-6)


def test_shuffled_string_order():
    """Strings in the order --shuffle leaves them: tables and sigma follow the given order."""
    rng = np.random.default_rng(9)
    L = 10
    a = _random_strings(L, 4, 50, rng)
    b = _random_strings(L, 4, 50, rng)
    perm_a, perm_b = rng.permutation(len(a)), rng.permutation(len(b))
    prob = _problem(L, 4, 4, [a[i] for i in perm_a], [b[i] for i in perm_b])
    _check_sigma(prob)


def test_wide_subspace_and_restart_limits():
    """The largest subspace (16 vectors, every compile-time residual/CGS size) and many restarts."""
    import sbd_tpb
    rng = np.random.default_rng(21)
    L = 12
    a = sorted(set([(1 << 5) - 1] + _random_strings(L, 5, 150, rng)))
    prob = _problem(L, 5, 5, a, a)
    h, s = _check_sigma(prob)
    e_or = s.davidson(max_it=30, max_nb=10, eps=1e-9)[0]
    r = h.davidson(sbd_tpb.default_params(max_it=20, max_nb=16, eps=1e-9), want_vector=False)
    assert r["energy"] == pytest.approx(e_or, abs=1e-8)
    r2 = h.davidson(sbd_tpb.default_params(max_it=400, max_nb=3, eps=1e-6), want_vector=False)
    assert r2["converged"] and r2["energy"] == pytest.approx(e_or, abs=1e-8)


def test_release_work_memory():
    """sbd_tpb_release_work gives back the Davidson vectors kept between solves and the sigma
    staging; the next solve allocates them again and gives the same answer."""
    import torch

    import sbd_tpb
    import synth
    prob = synth.make_problem("sci24", nstrings=1500)
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    p = sbd_tpb.default_params(max_it=20, max_nb=8, eps=1e-6)
    r1 = h.davidson(p, want_vector=False)
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    h.free_vectors()
    free_after, _ = torch.cuda.mem_get_info()
    # at least the 17 FP64 N-vectors of an 8-vector subspace (S, sigma(S), W)
    assert free_after - free_before >= 17 * prob.ndet * 8
    r2 = h.davidson(p, want_vector=False)
    assert r2["energy"] == r1["energy"] and r2["iterations"] == r1["iterations"]
    h.close()
