"""sbd_tpb_sigma_noalloc against the allocating sigma entry point (needs a B200).

The no-allocation entry point is for callers that cannot let the library cudaMalloc under them
(a code that has reserved the card's memory through its own pool, or one whose memory policy
forbids allocations after set-up); it stages C^T in a fixed 16 MiB device array of the library
instead.  This file is collected last so that, if it fails, a run that stops at the first
failure has already run every other test; it builds its own handles and passes alone or after
the other tests.
"""
import numpy as np
import pytest

from conftest import golden_problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["syn10_ab", "n2_1em3", "fci12"])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_noalloc_matches_sigma_device_twice(name, dtype):
    import torch

    import sbd_tpb
    prob, g, meta = golden_problem(name)
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    tdt = getattr(torch, dtype)
    # FP64 sigma agrees to rounding; the FP32 allocating path may take the split-BF16
    # tensor-core route for the alpha-beta term where this one uses the direct FP32 loop
    tol = 1e-12 if dtype == "float64" else 3e-5
    gen = torch.Generator(device="cuda").manual_seed(11)
    for call in range(2):  # two calls in a row share the scratch; each must be right
        x = torch.randn(prob.ndet, dtype=tdt, device="cuda", generator=gen)
        ref = torch.zeros_like(x)
        out = torch.full_like(x, float("nan"))
        h.sigma_device(x, ref)            # allocating entry point (separated convention)
        h.sigma_noalloc(x, out)           # no-allocation entry point, same convention
        torch.cuda.synchronize()
        err = float((out - ref).abs().max()) / float(ref.abs().max())
        assert err <= tol, (call, err)
    # accumulate: adds into the output like the other sigma entry points
    acc = ref.clone()
    h.sigma_noalloc(x, acc, accumulate=True)
    torch.cuda.synchronize()
    assert float((acc - 2 * ref).abs().max()) <= 2 * tol * float(ref.abs().max())
    h.close()


def test_noalloc_rejects_problems_beyond_scratch():
    import torch

    import sbd_tpb
    import synth
    prob = synth.make_problem("sci24", nstrings=1500)  # 2.25M determinants > 16 MiB of FP64
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    x = torch.zeros(prob.ndet, dtype=torch.float64, device="cuda")
    y = torch.zeros_like(x)
    with pytest.raises(sbd_tpb.TpbError) as e:
        h.sigma_noalloc(x, y)
    assert e.value.code == sbd_tpb.ERR_INVALID and "MiB scratch" in str(e.value)
    # the same problem in FP32 (9 MB of C^T) fits
    xf = torch.randn(prob.ndet, dtype=torch.float32, device="cuda")
    yf, rf = torch.zeros_like(xf), torch.zeros_like(xf)
    h.sigma_noalloc(xf, yf)
    h.sigma_device(xf, rf)
    torch.cuda.synchronize()
    assert float((yf - rf).abs().max()) <= 2e-5 * float(rf.abs().max())
    h.close()


def test_noalloc_call_allocates_nothing():
    """After the first call on the device (which looks up the scratch array's address and may
    load the library's device code), further calls leave the device's free memory and torch's
    allocations unchanged; the allocating entry point on the same handle does take memory (its
    C^T staging and work arrays), which shows the measurement sees an allocation."""
    import torch

    import sbd_tpb
    prob, g, meta = golden_problem("fci12")  # 853,776 determinants: 6.8 MB of FP64 C^T
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    gen = torch.Generator(device="cuda").manual_seed(5)
    x = torch.randn(prob.ndet, dtype=torch.float64, device="cuda", generator=gen)
    y = torch.zeros_like(x)
    ref = torch.zeros_like(x)
    h.sigma_noalloc(x, y)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    for _ in range(3):
        h.sigma_noalloc(x, y)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert torch.cuda.memory_allocated() == alloc0
    h.sigma_device(x, ref)
    torch.cuda.synchronize()
    free2, _ = torch.cuda.mem_get_info()
    assert free2 <= free1 - prob.ndet * 8, (free1, free2)
    assert float((y - ref).abs().max()) <= 1e-12 * float(ref.abs().max())
    h.close()


def test_noalloc_rejects_aliased_buffers():
    import torch

    import sbd_tpb
    prob, g, meta = golden_problem("syn10_ab")
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    x = torch.randn(prob.ndet, dtype=torch.float64, device="cuda")
    rc = sbd_tpb.lib().sbd_tpb_sigma_noalloc(h.h, x.data_ptr(), x.data_ptr(), 0, 0)
    assert rc == sbd_tpb.ERR_INVALID and b"distinct" in sbd_tpb.lib().sbd_tpb_last_error()
    with pytest.raises(sbd_tpb.TpbError):
        h.sigma_noalloc(x, x.to(torch.float32))
    h.close()
