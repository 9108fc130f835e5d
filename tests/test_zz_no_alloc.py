"""sbd_tpb_sigma_noalloc against the allocating sigma entry point (needs a B200).

The no-allocation entry point is for callers that cannot let the library cudaMalloc under them
(a caller that has reserved the card's memory through its own pool, or work issued inside
stream capture); it stages C^T in a fixed 16 MiB device array of the library instead.  This file
is collected last so that, if it fails, a run that stops at the first failure has already run
every other test; it builds its own handle and passes alone or after the other tests.
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
