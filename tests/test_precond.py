"""Learned Davidson preconditioner: oracle gradients pinned by finite differences (CPU), the
library's BF16 training kernels and fused inference kernel against the oracle, training on pairs
collected from plain Davidson runs, and the learned solve's answer against the FP64 one (GPU).

The network: x (64) -> 256 -> GELU -> 256 -> GELU -> y, correction t = d (1 + 0.5 tanh(y)); x depends only on
a determinant's spatial occupation, so y is the same across a spin-coupled set.
"""
import numpy as np
import pytest

from conftest import golden_problem

import pyoracle

H, F, WIN = 256, 64, 24
BOUND = 0.5  # correction factor 1 + BOUND tanh(y)


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def occ_window(s, nel):
    """Occupations of orbitals nel-12 .. nel+11 of string s (1 below orbital 0)."""
    bits = np.zeros(WIN, np.float32)
    for q in range(WIN):
        p = nel - WIN // 2 + q
        bits[q] = 1.0 if p < 0 else float((int(s) >> p) & 1) if p < 64 else 0.0
    return bits


def features(hdJ, e0, wa, wb):
    """Feature rows as the inference kernel forms them (before BF16 rounding): the spin-free
    diagonal, a zero residual slot, doubly and singly occupied windows."""
    x = np.zeros((len(hdJ), F), np.float32)
    x[:, 0] = np.arcsinh((hdJ - e0).astype(np.float32)) * np.float32(0.25)
    x[:, 2:2 + WIN] = wa * wb
    x[:, 2 + WIN:2 + 2 * WIN] = (wa + wb) % 2
    return x


def pair_of(i, j):
    return i * (i + 1) // 2 + j if i > j else j * (j + 1) // 2 + i


def exchange_sums(prob, strs):
    """Sum of (pq|qp) over the occupied pairs of each string."""
    L = prob.norb
    out = np.zeros(len(strs))
    for n, s in enumerate(strs):
        occ = [p for p in range(L) if (int(s) >> p) & 1]
        for a_ in range(len(occ)):
            for b_ in range(a_ + 1, len(occ)):
                pq = pair_of(occ[a_], occ[b_])
                out[n] += prob.eri_packed[pair_of(pq, pq)]
    return out


def np_forward64(x, W1, b1, W2, b2, w3, b3):
    k0, k1 = np.sqrt(2.0 / np.pi), 0.044715
    g = lambda z: 0.5 * z * (1.0 + np.tanh(k0 * (z + k1 * z ** 3)))
    a1 = g(x @ W1.T + b1)
    a2 = g(a1 @ W2.T + b2)
    return a2 @ w3 + b3[0]


def test_oracle_mlp_gradients_finite_difference():
    """orc_mlp_backward against central differences of an FP64 restatement of the loss."""
    rng = np.random.default_rng(5)
    n, din, dh = 9, 6, 5
    x = rng.normal(size=(n, din))
    a, b, w = rng.normal(size=n), rng.normal(size=n), rng.uniform(0.5, 2.0, size=n)
    P = [rng.normal(size=(dh, din)) * 0.5, rng.normal(size=dh) * 0.1, rng.normal(size=(dh, dh)) * 0.5,
         rng.normal(size=dh) * 0.1, rng.normal(size=dh) * 0.5, rng.normal(size=1) * 0.1]
    P = [bf16(p).astype(np.float64) for p in P]  # values exactly representable in FP32
    x = bf16(x).astype(np.float64)

    def loss(Q):
        y = np_forward64(x, *Q)
        return 0.5 * np.sum(w * (a * (1.0 + BOUND * np.tanh(y)) - b) ** 2) / n

    L_or, g_or = pyoracle.mlp_backward(x, a, b, w, *P)
    assert L_or == pytest.approx(loss(P), rel=1e-5)
    eps = 1e-6
    for t in range(6):
        fd = np.zeros_like(P[t])
        for idx in np.ndindex(P[t].shape):
            Qp = [q.copy() for q in P]
            Qm = [q.copy() for q in P]
            Qp[t][idx] += eps
            Qm[t][idx] -= eps
            fd[idx] = (loss(Qp) - loss(Qm)) / (2 * eps)
        np.testing.assert_allclose(g_or[t].reshape(fd.shape), fd, rtol=2e-4, atol=2e-6)


def random_params(rng, scale3=0.3):
    W1 = np.zeros((H, F), np.float32)
    W1[:, :2 + 2 * WIN] = rng.normal(0, np.sqrt(2 / 50), size=(H, 2 + 2 * WIN))
    b1 = rng.normal(0, 0.1, H)
    W2 = rng.normal(0, np.sqrt(2 / H), size=(H, H))
    b2 = rng.normal(0, 0.1, H)
    w3 = rng.normal(0, scale3 / np.sqrt(H), H)
    b3 = rng.normal(0, 0.05, 1)
    return [np.asarray(v, np.float32) for v in (W1, b1, W2, b2, w3, b3)]


def flat(P):
    return np.concatenate([p.ravel() for p in P]).astype(np.float32)


def rel_err(x, ref):
    return float(np.linalg.norm(x - ref) / max(np.linalg.norm(ref), 1e-300))


@pytest.mark.gpu
def test_gpu_mlp_gradients_vs_oracle():
    """BF16 tcgen05 forward/backward kernels against the CPU oracle on the same BF16 inputs."""
    import sbd_tpb
    rng = np.random.default_rng(11)
    P = random_params(rng)
    pc = sbd_tpb.Precond(0, seed=3)
    pc.set_params(flat(P))
    n = 384
    x = np.zeros((n, F), np.float32)
    x[:, 0] = rng.uniform(0, 1.5, n)
    x[:, 1] = rng.uniform(-1, 1, n)
    x[:, 2:2 + 2 * WIN] = rng.integers(0, 2, size=(n, 2 * WIN))
    x = bf16(x)
    a = rng.normal(size=n).astype(np.float32)
    b = (a * (1 + 0.3 * rng.normal(size=n))).astype(np.float32)
    w = rng.uniform(0.5, 2, n).astype(np.float32)
    grad, loss, y = pc.gradients(x, a, b, w)
    Pb = [bf16(P[0]), P[1], bf16(P[2]), P[3], P[4], P[5]]  # the kernels multiply BF16 weights
    y_ref = BOUND * np.tanh(pyoracle.mlp_forward(x, *Pb))
    L_ref, g_ref = pyoracle.mlp_backward(x, a, b, w, *Pb)
    # activations are BF16 on the tensor cores, FP32 in the oracle: errors of a few 1e-3
    assert np.max(np.abs(y - y_ref)) < 2e-2 * (1 + np.max(np.abs(y_ref)))
    assert loss == pytest.approx(L_ref, rel=2e-2)
    g = sbd_tpb.mlp_unpack(grad)
    names = ["W1", "b1", "W2", "b2", "w3", "b3"]
    for t in range(6):
        gr = np.asarray(g_ref[t]).reshape(np.shape(g[t]))
        if t == 0:  # only the 50 real inputs carry gradient
            gr, gt = gr[:, :50], g[t][:, :50]
            assert np.all(g[t][:, 50:] == 0)
        else:
            gt = g[t]
        e = rel_err(gt, gr)
        cos = float(np.dot(gt.ravel(), gr.ravel()) / (np.linalg.norm(gt) * np.linalg.norm(gr) + 1e-300))
        assert e < 4e-2 and cos > 0.999, (names[t], e, cos)


@pytest.mark.gpu
def test_gpu_mlp_inference_kernel_vs_oracle():
    """The fused per-determinant inference kernel (features in shared memory, two tcgen05 layers,
    GELU epilogues from TMEM) against features and forward pass restated on the CPU."""
    import sbd_tpb
    prob, _, _ = golden_problem("syn10_ab")
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    rng = np.random.default_rng(2)
    P = random_params(rng, scale3=0.5)
    pc = sbd_tpb.Precond(0, seed=4)
    pc.set_params(flat(P))
    n = prob.ndet
    hd = h.diagonal()
    e0 = float(hd.min()) - 0.3
    d = rng.normal(size=n) * np.exp(-0.3 * (hd - hd.min()))
    rnorm = 0.7
    t = pc.apply(h, d, e0, rnorm)
    na, nb = len(prob.astr), len(prob.bstr)
    nel_a = bin(int(prob.astr[0])).count("1")
    nel_b = bin(int(prob.bstr[0])).count("1")
    wa = np.array([occ_window(s, nel_a) for s in prob.astr])
    wb = np.array([occ_window(s, nel_b) for s in prob.bstr])
    hdJ = hd + np.repeat(exchange_sums(prob, prob.astr), nb) + np.tile(exchange_sums(prob, prob.bstr), na)
    x = features(hdJ, e0, np.repeat(wa, nb, axis=0), np.tile(wb, (na, 1)))
    Pb = [bf16(P[0]), P[1], bf16(P[2]), P[3], P[4], P[5]]
    y_ref = BOUND * np.tanh(pyoracle.mlp_forward(bf16(x), *Pb).astype(np.float64))
    y_gpu = t / np.where(d != 0, d, 1.0) - 1.0
    assert np.max(np.abs(y_gpu - y_ref)) < 2e-2 * (1 + np.max(np.abs(y_ref)))
    # the same network through the training kernels gives the same y
    _, _, y_train = pc.gradients(bf16(x), np.ones(n, np.float32), np.ones(n, np.float32),
                                 np.ones(n, np.float32))
    assert np.max(np.abs(y_gpu - y_train)) < 1e-2 * (1 + np.max(np.abs(y_ref)))
    h.close()


@pytest.mark.gpu
def test_gpu_mlp_inference_budgeted_subset():
    """Beyond 2^22 determinants the inference kernel corrects only |d_i| >= |d| / 2^11 (gathered by
    index); the other entries keep the diagonal correction exactly."""
    import sbd_tpb
    import synth
    prob = synth.make_problem("sci24")  # 16M determinants
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    rng = np.random.default_rng(8)
    P = random_params(rng, scale3=0.5)
    pc = sbd_tpb.Precond(0, seed=5)
    pc.set_params(flat(P))
    n = prob.ndet
    hd = h.diagonal()
    d = rng.standard_cauchy(size=n) * 1e-3  # heavy-tailed: a few large entries
    e0, rnorm = float(hd.min()) - 0.2, 1.3
    t = pc.apply(h, d, e0, rnorm)
    theta = np.sqrt(np.dot(d, d) / (1 << 22))
    big = np.abs(d) >= theta * (1 + 1e-9)       # away from the threshold on both sides: the
    small = np.abs(d) < theta * (1 - 1e-9)      # library sums |d|^2 in another order
    assert 0 < big.sum() <= (1 << 22)
    assert np.array_equal(t[small], d[small])
    # the corrected entries agree with the training forward pass on the same features
    sel = np.flatnonzero(big)[:2048]
    nb = len(prob.bstr)
    nel = bin(int(prob.astr[0])).count("1")
    wa = np.array([occ_window(prob.astr[i // nb], nel) for i in sel])
    wb = np.array([occ_window(prob.bstr[i % nb], nel) for i in sel])
    kxa = exchange_sums(prob, prob.astr[sel // nb])
    kxb = exchange_sums(prob, prob.bstr[sel % nb])
    x = features(hd[sel] + kxa + kxb, e0, wa, wb)
    one = np.ones(len(sel), np.float32)
    _, _, y_train = pc.gradients(bf16(x), one, one, one)
    y_gpu = t[sel] / d[sel] - 1.0
    assert np.max(np.abs(y_gpu - y_train)) < 1e-2 * (1 + np.max(np.abs(y_train)))
    h.close()


@pytest.fixture(scope="module")
def trained():
    """A preconditioner trained on pairs of the plain FP64 Davidson on the 12-orbital full CI
    problem; held-out pairs from the 24-orbital selected-CI problem."""
    import sbd_tpb
    import synth
    pc = sbd_tpb.Precond(0, seed=7)
    h = sbd_tpb.Handle(0)
    h.set_problem(synth.make_problem("fci12"))
    e_train = pc.collect(h, sbd_tpb.default_params(max_it=30, max_nb=10, eps=1e-9),
                         samples_per_step=1 << 15, role=0)
    h.close()
    h2 = sbd_tpb.Handle(0)
    h2.set_problem(synth.make_problem("sci24"))
    pc.collect(h2, sbd_tpb.default_params(max_it=30, max_nb=10, eps=1e-8),
               samples_per_step=1 << 15, role=1)
    h2.close()
    before = pc.evaluate(0)
    held_before = pc.evaluate(1)
    loss = pc.train(epochs=4, batch=8192, lr=1e-3)
    # one more round on pairs from the learned solver's own trajectory
    h = sbd_tpb.Handle(0)
    h.set_problem(synth.make_problem("fci12"))
    pc.collect(h, sbd_tpb.default_params(max_it=30, max_nb=10, eps=1e-8,
                                         preconditioner=sbd_tpb.PRECOND_LEARNED),
               samples_per_step=1 << 15, role=0)
    h.close()
    loss = pc.train(epochs=2, batch=8192, lr=1e-3)
    return dict(pc=pc, e_train=e_train, before=before, held_before=held_before, loss=loss)


@pytest.mark.gpu
def test_gpu_precond_training_gain(trained):
    """Training lowers the error of the correction against the exact one (Psi - W_k, fitted in
    scale) on its training pairs and reports the held-out change."""
    pc = trained["pc"]
    assert pc.num_samples(0) > 10000 and pc.num_samples(1) > 10000
    l0, d0 = trained["before"]
    assert l0 == pytest.approx(d0, rel=1e-6)  # untrained network == diagonal correction
    lt, dt = pc.evaluate(0)
    lh, dh = pc.evaluate(1)
    print(f"\ntraining pairs: learned/diagonal error {lt / dt:.4f}; held-out (sci24): {lh / dh:.4f}")
    assert lt < 0.95 * dt
    assert lh < dh  # held-out pairs of another system (never trained on) improve too


@pytest.mark.gpu
def test_gpu_davidson_learned_same_answer(trained):
    """The learned correction changes the iteration count, never the answer: FP64 and mixed
    solves with the trained network reach the plain FP64 energy."""
    import sbd_tpb
    import synth
    prob = synth.make_problem("fci12")
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    r64 = h.davidson(sbd_tpb.default_params(max_it=40, max_nb=10, eps=1e-5), want_vector=False)
    h.set_preconditioner(trained["pc"])
    rl = h.davidson(sbd_tpb.default_params(max_it=40, max_nb=10, eps=1e-5,
                                           preconditioner=sbd_tpb.PRECOND_LEARNED), want_vector=False)
    rm = h.davidson(sbd_tpb.default_params(max_it=40, max_nb=10, eps=1e-5, precision=sbd_tpb.MIXED,
                                           preconditioner=sbd_tpb.PRECOND_LEARNED), want_vector=False)
    print(f"\nfci12 to |r| < 1e-5: diagonal {r64['iterations']} steps, learned {rl['iterations']} steps "
          f"({rl['learned_steps']} learned, {rl['fallback_steps']} fallbacks); mixed+learned "
          f"{rm['iterations']} steps")
    assert r64["converged"] and rl["converged"] and rm["converged"]
    assert rl["learned_steps"] > 0 and rm["learned_steps"] > 0
    # |r| < 1e-5 bounds the energy error by ~|r|^2 / gap
    assert abs(rl["energy"] - r64["energy"]) < 1e-7
    assert abs(rm["energy"] - r64["energy"]) < 1e-6
    h.close()


@pytest.mark.gpu
def test_gpu_learned_held_out_solver_steps(trained):
    """Solver steps on a system the network never saw (24 orbitals, 2,000 x 2,000 selected
    strings), learned against diagonal correction, FP64 and mixed, to |r| < 1e-5.  Printed for the
    record; asserted: the same energy, the network was used, and a learned solve takes at most 2x
    the diagonal solve's steps.  On these random-integral Hamiltonians the learned correction does
    not reliably save steps, and the step counts of either correction move by up to ~30 % with
    last-bit changes of the arithmetic (learned / diagonal measured 0.9-1.6 here), so the bound only
    catches a learned correction that derails the solve."""
    import sbd_tpb
    import synth
    h = sbd_tpb.Handle(0)
    h.set_problem(synth.make_problem("sci24", nstrings=2000))
    h.set_preconditioner(trained["pc"])
    res = {}
    for prec, tag in ((sbd_tpb.FP64, "fp64"), (sbd_tpb.MIXED, "mixed")):
        for pre, ptag in ((sbd_tpb.PRECOND_DIAGONAL, "diagonal"), (sbd_tpb.PRECOND_LEARNED, "learned")):
            res[tag, ptag] = h.davidson(sbd_tpb.default_params(max_it=40, max_nb=8, eps=1e-5, precision=prec,
                                                               preconditioner=pre), want_vector=False)
    print("\nheld-out sci24 (2000 x 2000) steps to |r| < 1e-5: " + ", ".join(
        f"{t}/{p} {r['iterations']} ({r['learned_steps']} learned, {r['fallback_steps']} fallbacks)"
        for (t, p), r in res.items()))
    e = res["fp64", "diagonal"]["energy"]
    for (t, p), r in res.items():
        assert r["converged"], (t, p)
        assert abs(r["energy"] - e) < 1e-6, (t, p, r["energy"], e)
    for t in ("fp64", "mixed"):
        assert res[t, "learned"]["learned_steps"] > 0
        assert res[t, "learned"]["iterations"] <= 2 * res[t, "diagonal"]["iterations"]
    h.set_preconditioner(None)
    h.close()


@pytest.mark.gpu
def test_gpu_learned_requires_attached_model():
    import sbd_tpb
    prob, _, _ = golden_problem("syn10_ab")
    h = sbd_tpb.Handle(0)
    h.set_problem(prob)
    with pytest.raises(sbd_tpb.TpbError):
        h.davidson(sbd_tpb.default_params(preconditioner=sbd_tpb.PRECOND_LEARNED), want_vector=False)
    h.close()
