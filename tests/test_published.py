"""Energies the reference publishes for its own data sets (data/h2o/README.md:7-10,
data/n2/README.md:7-12: 8 decimals, from 4.1e5 to 6.3e8 determinants), reproduced by the library.

The string sets are in tests/golden/published.npz (read from the reference's data files by the
oracle's LoadAlphaDets restatement; tests/golden/make_golden.py), the Hamiltonians are those of the
h2o_1em3 / n2_1em3 fixtures (the same FCIDUMP files).  FP64 solves must land within 1e-8 Ha of the
published value (its rounding is 5e-9); mixed-precision solves within 1e-6 Ha.

The h2o sets above 1e-5 are dense (25,062 of the 42,504 possible strings at 1e-7, about a thousand
doubles per string), so their solves take a minute or more on one B200 (1e-6 FP64 113 s, 1e-6 mixed
55 s, 1e-7 mixed 399 s); the 1e-7 set (6.3e8 determinants) runs only with SBD_TPB_LONG_TESTS=1."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_cases, load_golden

PUB = golden_cases()["published"]
README_COUNTS = {  # strings per the READMEs' tables
    "h2o_1em4": 1543, "h2o_1em5": 5514, "h2o_1em6": 13822, "h2o_1em7": 25062,
    "n2_3em4": 642, "n2_1em4": 1387, "n2_1em5": 4041, "n2_1em6": 9332,
}


def _strings(name):
    return np.load(os.path.join(GOLDEN, "published.npz"))[f"{name}_astr"]


def published_problem(name):
    from sbd_tpb import Problem
    meta = PUB[name]
    base = load_golden(meta["base"])
    L = golden_cases()[meta["base"]]["norb"]
    a = _strings(name)
    return Problem(norb=L, nelec=2 * bin(int(a[0])).count("1"), core=float(base["core"][0]),
                   h1=base["h1"], eri_packed=base["eri"], astr=a, bstr=a.copy()), meta


@pytest.mark.parametrize("name", sorted(PUB))
def test_published_fixture(name):
    """Sorted, unique, the READMEs' string counts, every string with the base case's electron count."""
    a = _strings(name)
    assert len(a) == README_COUNTS[name] == PUB[name]["na"]
    assert np.all(np.diff(a.astype(np.uint64)) > 0)
    base = load_golden(PUB[name]["base"])
    ne = bin(int(base["astr"][0])).count("1")
    assert all(bin(int(s)).count("1") == ne for s in a)
    assert int(a.max()) < (1 << golden_cases()[PUB[name]["base"]]["norb"])


def test_oracle_published_energy_n2_3em4():
    """The oracle's own Davidson (one core, ~40 s) on the 412,164-determinant n2 set reproduces the
    published energy: the CPU restatement is pinned at a second, larger size of the reference's data."""
    import pyoracle
    prob, meta = published_problem("n2_3em4")
    ham = pyoracle.Hamiltonian.from_arrays(prob.norb, prob.nelec, prob.core, prob.h1, prob.eri_packed)
    e, W, ns, resid = pyoracle.System(ham, prob.astr, prob.bstr).davidson(max_it=10, max_nb=10, eps=1e-6)
    assert resid < 1e-6
    assert e == pytest.approx(meta["published"], abs=1e-8)


def _solve(prob, precision, eps):
    import sbd_tpb
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    r = h.davidson(sbd_tpb.default_params(max_it=60, max_nb=10, eps=eps, precision=precision),
                   want_vector=False)
    h.close()
    return r


LONG = pytest.mark.skipif(os.environ.get("SBD_TPB_LONG_TESTS") != "1",
                          reason="minutes-long solve; set SBD_TPB_LONG_TESTS=1")


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["n2_3em4", "n2_1em4", "n2_1em5", "n2_1em6", "h2o_1em4", "h2o_1em5",
                                  "h2o_1em6"])
def test_gpu_published_energy_fp64(name):
    import sbd_tpb
    prob, meta = published_problem(name)
    r = _solve(prob, sbd_tpb.FP64, 1e-6)
    assert r["converged"]
    assert r["energy"] == pytest.approx(meta["published"], abs=1e-8)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["h2o_1em5", "h2o_1em6", pytest.param("h2o_1em7", marks=LONG)])
def test_gpu_published_energy_mixed(name):
    """FP32 vectors, FP64 projections and a final FP64 sigma (3.0e7 and 1.9e8 determinants; 6.3e8 with
    SBD_TPB_LONG_TESTS=1)."""
    import sbd_tpb
    prob, meta = published_problem(name)
    r = _solve(prob, sbd_tpb.MIXED, 1e-5)
    assert r["converged"]
    assert r["energy"] == pytest.approx(meta["published"], abs=1e-6)


@pytest.mark.gpu
def test_gpu_sigma_dense_singles(oracle):
    """Sigma where the alpha-beta kernel's beta program is split by ket range (dense beta singles: n2 1e-5,
    4,041 strings, 1.6e7 determinants, tens of singles per string): the general form equals the oracle's
    sigma (orc_sigma_rows, the reference's convention and per-element order) at 200 sampled determinants,
    FP64 within 1e-12 and FP32 within 2e-5 of the largest sampled |sigma|; and the exchange-symmetric
    form (its alpha-beta term on the upper triangle only) equals the general form on a symmetric vector
    (FP64 1e-13, FP32 3e-6 of the largest |sigma|)."""
    import torch

    import sbd_tpb
    from test_large_configs import _hash_vector_device
    prob, meta = published_problem("n2_1em5")
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    rows = np.random.default_rng(6).choice(prob.ndet, size=200, replace=False)
    ham = oracle.Hamiltonian.from_arrays(prob.norb, prob.nelec, prob.core, prob.h1, prob.eri_packed)
    ref = oracle.System(ham, prob.astr, prob.bstr).sigma_rows(rows)  # closed-form hash vector
    scale = float(np.max(np.abs(ref)))
    idx = torch.from_numpy(rows.astype(np.int64)).cuda()
    x64 = _hash_vector_device(prob.ndet)
    for x, tol in ((x64, 1e-12), (x64.float(), 2e-5)):
        y = torch.empty_like(x)
        h.sigma_device(x, y, separated=False)
        assert np.max(np.abs(y[idx].double().cpu().numpy() - ref)) <= tol * scale, (x.dtype, tol)
        del y
    del x64
    n = len(prob.astr)
    g = torch.Generator(device="cuda").manual_seed(8)
    r = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
    xs = ((r + r.T) * 0.5).reshape(-1).contiguous()
    del r
    for x, tol in ((xs, 1e-13), (xs.float(), 3e-6)):
        gen, sym = torch.empty_like(x), torch.empty_like(x)
        h.sigma_device(x, gen)
        h.sigma_device(x, sym, symmetric=True)
        err = float((sym.double() - gen.double()).abs().max()) / float(gen.double().abs().max())
        assert err <= tol, (x.dtype, err)
        del gen, sym
    h.close()
