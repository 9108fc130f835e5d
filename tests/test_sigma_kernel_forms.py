"""Every kernel form of sigma gives the same bits (needs a B200).

Vectors whose rows are 16-byte aligned (row length a multiple of 16 bytes / element size, base
address 16-byte aligned) take the passes that cover two 16-byte column groups per thread; a vector
viewed one element into its buffer takes the one-group passes with scalar loads.  Both sum the same
terms in the same order with the same roundings (fused multiply-add for the doubles terms, rounded
FP64 products for the singles and the diagonal), so sigma is bitwise equal: general form
(convention 1, with and without accumulate) and exchange-symmetric one-pass form (convention 2)."""
import pytest

from conftest import golden_problem

pytestmark = pytest.mark.gpu


def _vec(n, dtype, seed, symmetric):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    r = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
    if symmetric:
        r = (r + r.T) * 0.5
    return r.to(dtype).reshape(-1).contiguous()


def _offset_copy(v):
    """v copied into a buffer one element longer and viewed from its second element: same values,
    contiguous, but not 16-byte aligned."""
    import torch
    buf = torch.empty(v.numel() + 1, dtype=v.dtype, device=v.device)
    view = buf[1:]
    view.copy_(v)
    assert view.data_ptr() % 16 != 0
    return view


def _problems():
    import synth
    yield "fci12", golden_problem("fci12")[0]
    yield "sci24", synth.make_problem("sci24", nstrings=1500)


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_aligned_and_offset_vectors_give_same_bits(dtype):
    import torch

    import sbd_tpb
    tdt = getattr(torch, dtype)
    vw = 16 // torch.empty(0, dtype=tdt).element_size()
    for name, prob in _problems():
        n = len(prob.astr)
        assert n % vw == 0, name  # aligned rows: the two-group passes run
        h = sbd_tpb.Handle(0)
        h.set_problem(prob)
        for symmetric in (False, True):
            x = _vec(n, tdt, 5, symmetric)
            y0 = _vec(n, tdt, 6, False)
            for accumulate in ((False,) if symmetric else (False, True)):
                a_out = y0.clone()
                h.sigma_device(x, a_out, accumulate=accumulate, symmetric=symmetric)
                u_x, u_out = _offset_copy(x), _offset_copy(y0)
                h.sigma_device(u_x, u_out, accumulate=accumulate, symmetric=symmetric)
                torch.cuda.synchronize()
                assert torch.isfinite(a_out).all()
                assert torch.equal(a_out, u_out), (name, dtype, symmetric, accumulate,
                                                   float((a_out.double() - u_out.double()).abs().max()))
        h.close()
