"""The learned planner: the FP64 oracle of the network (finite differences), the problem generator, the model text
and host evaluation through the C ABI (CPU), and the device training kernels against the oracle (GPU)."""

from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import mlp as omlp

D, H = 32, 64


def _params(seed=3, d=D, h=H):
    from crd_b200.learned_planner import init_params

    p = init_params(d, h, seed).astype(np.float64)
    rng = np.random.default_rng(seed)
    # non-zero biases so every parameter's gradient is exercised
    p += rng.normal(scale=0.05, size=p.shape)
    return p


def _data(rows=300, seed=5, d=D):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(rows, d))
    t = np.sin(x[:, 0]) + 0.5 * x[:, 1] * x[:, 2] - 0.2 * x[:, 3]
    return x, t


def test_oracle_gradient_matches_finite_differences():
    d, h = 6, 8
    p = _params(d=d, h=h)
    x, t = _data(40, d=d)
    _, g = omlp.loss_and_grad(p, x, t, d, h)
    eps = 1e-6
    for i in range(p.size):
        e = np.zeros_like(p)
        e[i] = eps
        lp, _ = omlp.loss_and_grad(p + e, x, t, d, h)
        lm, _ = omlp.loss_and_grad(p - e, x, t, d, h)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 * (1 + abs(fd)), f"param {i}: fd {fd} vs {g[i]}"


def test_problem_generator_follows_its_contract():
    from crd_b200.learned_planner import MAX_INPUT_BYTES, problems, smooth7
    from crd_b200._lib import R2C

    assert len(smooth7(64, 1 << 22)) == 1745  # the 7-smooth candidates in [64, 2^22]
    probs = problems(400, seed=11)
    assert probs == problems(400, seed=11)
    ok = set(smooth7(16, 1 << 22))
    for pr in probs:
        pts = int(np.prod(pr.dims))
        for dd in pr.dims:
            assert dd in ok
        if len(pr.dims) == 1:
            assert 64 <= pts <= 1 << 22
        if pr.kind == R2C:
            assert pr.dims[-1] % 2 == 0
            assert len(pr.dims) == 1 or not pr.padded  # 2-D real plans take packed batches
        elem = 4 if pr.kind == R2C else 8
        assert 1 <= pr.batch <= 65536 and pr.batch * (pts + 8) * elem <= MAX_INPUT_BYTES
    kinds = {(len(p.dims), p.kind) for p in probs}
    assert len(kinds) == 4
    assert any(p.padded for p in probs) and any(not p.padded for p in probs)


def test_log_parser_groups_passes():
    from crd_b200.learned_planner import parse_log

    f = ",".join(["1"] * D)
    text = (f"k1 pipelined=0 P=16 lpc=1 lines=8 ms=0.5 feat={f}\n"
            f"k1 pipelined=0 P=32 lpc=1 lines=8 ms=0.25 feat={f} best heur\n"
            f"k1 pipelined=1 P=16 lpc=2 lines=8 ms=-1.000000 feat={f}\n"
            f"k2 pipelined=0 P=16 lpc=4 lines=8 ms=0.125 feat={f} best\n")
    g = parse_log(text)
    assert [x.key for x in g] == ["k1", "k2"]
    assert g[0].ms.tolist() == [0.5, 0.25] and g[0].best == 1 and g[0].heur == 1
    assert g[1].heur == -1 and g[1].feats.shape == (1, D)


def test_log_parser_separates_decompositions():
    """Decomposition lines (" decomp ") and launch-shape lines of one log go to separate groups."""
    from crd_b200.learned_planner import parse_log

    f = ",".join(["1"] * D)
    text = (f"D|dev|n1048576:b8:u1:p0:x0 decomp kind=3 n1=1024 batch=256 ms=2.5 feat={f} heur\n"
            f"D|dev|n1048576:b8:u1:p0:x0 decomp kind=3 n1=512 batch=256 ms=2.25 feat={f} best\n"
            f"k1 pipelined=0 P=16 lpc=1 lines=8 ms=0.5 feat={f} best\n")
    d = parse_log(text, decomp=True)
    p = parse_log(text)
    assert len(d) == 1 and d[0].best == 1 and d[0].heur == 0 and d[0].ms.tolist() == [2.5, 2.25]
    assert len(p) == 1 and p[0].key == "k1"


def test_two_models_in_one_text():
    """A model text may hold the launch-shape model and the decomposition model; the library imports both and
    exports both, and the decomposition model alone keeps the shape model already loaded."""
    import crd_b200.hesap as F
    from crd_b200.learned_planner import DECOMP_TAG, Model

    rng = np.random.default_rng(3)
    p = _params().astype(np.float32)
    a = Model(rng.normal(size=D).astype(np.float32), rng.uniform(0.5, 2, size=D).astype(np.float32), -1.0, 2.0, p)
    b = Model(a.mean, a.std, 0.5, 1.5, (p * 0.5).astype(np.float32), tag=DECOMP_TAG)
    try:
        F.learned_model_import(a.text() + b.text())
        got = Model.parse_all(F.learned_model_export())
        assert [m.tag for m in got] == ["crdfft-mlp", DECOMP_TAG]
        assert np.array_equal(got[1].params, b.params) and got[1].t_mean == b.t_mean
        F.learned_model_forget()
        F.learned_model_import(a.text())
        F.learned_model_import(b.text())
        assert [m.tag for m in Model.parse_all(F.learned_model_export())] == ["crdfft-mlp", DECOMP_TAG]
    finally:
        F.learned_model_forget()


def test_model_text_round_trip_and_host_predict():
    """The library parses the model text, exports it unchanged, rejects malformed texts, and its host forward pass
    agrees with the FP64 oracle."""
    import crd_b200.hesap as F
    from crd_b200._lib import CrdFftError, lib
    from crd_b200.learned_planner import Model

    assert lib().crdfft_pass_feature_count() == D
    rng = np.random.default_rng(2)
    p = _params().astype(np.float32)
    m = Model(rng.normal(size=D).astype(np.float32), rng.uniform(0.5, 2, size=D).astype(np.float32), -1.5, 2.0, p)
    F.learned_model_import(m.text())
    try:
        back = Model.parse(F.learned_model_export())
        assert np.array_equal(back.params, m.params) and np.array_equal(back.mean, m.mean)
        for _ in range(5):
            f = rng.normal(size=D).astype(np.float32)
            want, _ = omlp.forward(p, ((f - m.mean) / m.std)[None, :], D, H)
            got = F.learned_predict(f)
            assert abs(got - (m.t_mean + m.t_std * want[0])) <= 1e-4 * (1 + abs(got))
        bad = m.text().replace("params", "parms")
        with pytest.raises(CrdFftError):
            F.learned_model_import(bad)
        with pytest.raises(CrdFftError):
            F.learned_model_import(m.text().replace("dims 32", "dims 31"))
        assert Model.parse(F.learned_model_export()).params.size == p.size  # the good model is kept
    finally:
        F.learned_model_forget()


# ---- device kernels ------------------------------------------------------------------------------------------


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def _grads(p, x, t, d=D, h=H):
    import torch

    from crd_b200._lib import check, lib

    L = lib()
    P, X, T = _dev(p), _dev(x), _dev(t)
    G = torch.empty_like(P)
    loss = torch.zeros(1, device="cuda")
    W = torch.empty(L.crdfft_mlp_workspace_floats(d, h, x.shape[0]), device="cuda")
    check(L.crdfft_mlp_gradients(d, h, P.data_ptr(), X.data_ptr(), T.data_ptr(), x.shape[0], G.data_ptr(),
                                 loss.data_ptr(), W.data_ptr(), None), "grad")
    torch.cuda.synchronize()
    return float(loss.item()), G.cpu().numpy()


@pytest.mark.gpu
def test_device_gradients_match_oracle():
    p = _params()
    x, t = _data(5000)
    loss, g = _grads(p, x, t)
    lo, go = omlp.loss_and_grad(p.astype(np.float32), x.astype(np.float32), t.astype(np.float32), D, H)
    assert abs(loss - lo) <= 1e-5 * (1 + lo)
    err = np.linalg.norm(g - go) / np.linalg.norm(go)
    assert err <= 1e-5, f"gradient rel-L2 {err:.2e}"
    assert np.max(np.abs(g - go)) <= 1e-4 * (1 + np.max(np.abs(go)))


@pytest.mark.gpu
def test_device_forward_matches_oracle_and_is_deterministic():
    import torch

    from crd_b200.learned_planner import Model, predict_device

    p = _params().astype(np.float32)
    x, _ = _data(777)
    m = Model(np.zeros(D, np.float32), np.ones(D, np.float32), 0.0, 1.0, p)
    y = predict_device(m, x.astype(np.float32))
    yo, _ = omlp.forward(p, x.astype(np.float32), D, H)
    assert np.max(np.abs(y - yo)) <= 1e-4 * (1 + np.max(np.abs(yo)))
    _, g1 = _grads(p, x, np.zeros(777))
    _, g2 = _grads(p, x, np.zeros(777))
    assert np.array_equal(g1, g2)  # fixed-order reductions: bit-identical reruns
    torch.cuda.synchronize()


@pytest.mark.gpu
def test_device_adam_matches_oracle():
    import torch

    from crd_b200._lib import check, lib

    rng = np.random.default_rng(9)
    n = 5000
    p, g = rng.normal(size=n), rng.normal(size=n)
    m, v = rng.normal(scale=0.1, size=n), rng.uniform(0, 0.1, size=n)
    P, G, M, V = (_dev(a) for a in (p, g, m, v))
    check(lib().crdfft_mlp_adam(P.data_ptr(), G.data_ptr(), M.data_ptr(), V.data_ptr(), n, 7, 1e-3, 0.9, 0.999,
                                1e-8, None), "adam")
    torch.cuda.synchronize()
    po, mo, vo = omlp.adam(p.astype(np.float32).astype(np.float64), g.astype(np.float32), m.astype(np.float32),
                           v.astype(np.float32), 7, 1e-3)
    assert np.max(np.abs(P.cpu().numpy() - po)) <= 1e-6
    assert np.max(np.abs(M.cpu().numpy() - mo)) <= 1e-6
    assert np.max(np.abs(V.cpu().numpy() - vo)) <= 1e-6


@pytest.mark.gpu
def test_training_fits_a_smooth_target():
    from crd_b200.learned_planner import predict_device, train

    x, t = _data(4000)
    model, hist = train(x.astype(np.float32), t.astype(np.float32), steps=600, lr=3e-3, log_every=100)
    assert hist[-1][1] < 0.25 * hist[0][1]
    xv, tv = _data(1000, seed=6)
    pred = predict_device(model, xv.astype(np.float32))
    assert np.sqrt(np.mean((pred - tv) ** 2)) < 0.5 * np.std(tv)


@pytest.mark.gpu
def test_measure_log_carries_features_and_learned_mode_plans_correctly():
    """The measuring planner's log has a 32-feature vector per candidate; a plan created in learned mode (from the
    committed model when present, else one trained here on those timings) computes the right transform."""
    import os

    import torch

    import crd_b200 as cf
    import crd_b200.hesap as F
    from crd_b200.learned_planner import Model, dataset, collect, problems, train

    ms = collect(problems(12, seed=21))
    assert sum(len(m.groups) for m in ms) >= 12
    for m in ms:
        for g in m.groups:
            assert g.feats.shape[1] == D and np.all(g.ms > 0)
    path = os.path.join(os.path.dirname(cf.__file__), "data", "planner_mlp_b200.txt")
    if os.path.exists(path):
        with open(path) as f:
            model = Model.parse(f.read())
    else:
        x, y = dataset(ms)
        model, _ = train(x, y, steps=200)
    F.learned_model_import(model.text())
    F.set_planner("learned")
    try:
        F.wisdom_forget()
        for n, batch in ((4096, 33), (65536, 3), (1000, 17)):
            x = (torch.rand(batch, n, 2) * 2 - 1).view(torch.complex64).view(batch, n).cuda()
            o = torch.empty_like(x)
            cf.Plan([n], batch=batch).execute(x, o)
            torch.cuda.synchronize()
            want = np.fft.fft(x.cpu().numpy().astype(np.complex128), axis=1)
            got = o.cpu().numpy()
            assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-6
    finally:
        F.set_planner("estimate")
        F.learned_model_forget()
        F.wisdom_forget()
