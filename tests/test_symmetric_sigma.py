"""The one-pass sigma for exchange-symmetric vectors (sbd_tpb_sigma_device, convention 2) against
the general two-pass sigma (convention 1) on symmetric vectors (needs a B200).

With identical alpha and beta string lists and C[Ia, Ib] = C[Ib, Ia] the beta part of sigma is
the transpose of the alpha part (the reference computes both, tpb/mult.h:717-790), so the library
runs one gathering pass that writes B = H_ii C / 2 + (alpha part) and forms sigma = B + B^T.
Davidson started from the HF determinant stays in that sector and uses it.
"""
import numpy as np
import pytest

from conftest import golden_problem

pytestmark = pytest.mark.gpu


def _symmetric(n, dtype, seed):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    r = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
    return ((r + r.T) * 0.5).to(dtype).reshape(-1).contiguous()


@pytest.mark.parametrize("name", ["fci12", "n2_1em3", "h2o_1em3"])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_symmetric_sigma_matches_general(name, dtype):
    import torch

    import sbd_tpb
    prob, g, meta = golden_problem(name)
    assert np.array_equal(prob.astr, prob.bstr)
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    tdt = getattr(torch, dtype)
    # FP64: both are FP64 sums of the same terms in different orders; FP32: FP32 vectors and
    # values (the alpha-beta term is the same kernel in both)
    tol = 1e-13 if dtype == "float64" else 3e-6
    n = len(prob.astr)
    for seed in (1, 2):
        x = _symmetric(n, tdt, seed)
        ref, out = torch.zeros_like(x), torch.full_like(x, float("nan"))
        h.sigma_device(x, ref)
        h.sigma_device(x, out, symmetric=True)
        torch.cuda.synchronize()
        err = float((out.double() - ref.double()).abs().max()) / float(ref.double().abs().max())
        assert err <= tol, (name, dtype, seed, err)
    h.close()


def test_symmetric_sigma_larger_selected_set():
    """24 orbitals, 1500 selected strings per spin (2.25M determinants): sparse alpha-beta kernel,
    block shapes with partial slabs."""
    import torch

    import sbd_tpb
    import synth
    prob = synth.make_problem("sci24", nstrings=1500)
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    x = _symmetric(len(prob.astr), torch.float64, 3)
    ref, out = torch.zeros_like(x), torch.zeros_like(x)
    h.sigma_device(x, ref)
    h.sigma_device(x, out, symmetric=True)
    torch.cuda.synchronize()
    assert float((out - ref).abs().max()) <= 1e-13 * float(ref.abs().max())
    h.close()


def test_symmetric_sigma_needs_identical_strings():
    import torch

    import sbd_tpb
    prob, g, meta = golden_problem("syn10_ab")  # distinct alpha / beta lists
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    x = torch.zeros(prob.ndet, dtype=torch.float64, device="cuda")
    y = torch.zeros_like(x)
    with pytest.raises(sbd_tpb.TpbError) as e:
        h.sigma_device(x, y, symmetric=True)
    assert e.value.code == sbd_tpb.ERR_STATE
    with pytest.raises(sbd_tpb.TpbError) as e:
        h.sigma_device(x, y, accumulate=True, symmetric=True)
    assert e.value.code == sbd_tpb.ERR_INVALID
    h.close()
