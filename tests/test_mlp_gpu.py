"""GPU checks of the proposal network against its CPU oracle
(oracle/mlp_oracle.py): the tensor-core GEMM, the forward pass, the
gradients of every parameter block, and Adam training."""

import ctypes as C

import numpy as np
import pytest

from bmmpy_b200 import _native as N
from oracle import mlp_oracle as O

pytestmark = pytest.mark.gpu


def _gemm(A, B):
    A = np.ascontiguousarray(A, np.float32)
    B = np.ascontiguousarray(B, np.float32)
    Cm = np.zeros((A.shape[0], B.shape[0]), np.float32)
    N.check(N.lib().bmm_mlp_gemm(N.f32p(A), N.f32p(B), A.shape[0], B.shape[0], A.shape[1],
                                 N.f32p(Cm)))
    return Cm


@pytest.mark.parametrize("M,Nn,K", [(128, 256, 64), (1, 7, 5), (300, 256, 512), (513, 300, 130),
                                    (256, 512, 1000)])
def test_tensor_core_gemm_matches_bf16_product(M, Nn, K):
    rng = np.random.default_rng(M * 7 + Nn + K)
    A = rng.standard_normal((M, K)).astype(np.float32)
    B = rng.standard_normal((Nn, K)).astype(np.float32)
    got = _gemm(A, B)
    want = O.bf16(A).astype(np.float64) @ O.bf16(B).astype(np.float64).T
    # FP32 accumulation of exact BF16 products
    assert np.allclose(got, want, rtol=1e-4, atol=1e-4 * np.sqrt(K))


@pytest.fixture()
def net():
    h = C.c_void_p()
    N.check(N.lib().bmm_mlp_create(5, 1e-3, C.byref(h)))
    yield h
    N.lib().bmm_mlp_destroy(h)


def _params(h):
    p = np.zeros(O.N_PARAMS, np.float32)
    N.check(N.lib().bmm_mlp_get_params(h, N.f32p(p)))
    return p


def _inputs(rows, seed):
    rng = np.random.default_rng(seed)
    X = np.concatenate([rng.standard_normal((rows, 256)),
                        rng.choice([-1.0, 1.0], (rows, 256))], axis=1).astype(np.float32)
    T = rng.random((rows, 256)) ** 8
    T = (T / T.sum(axis=1, keepdims=True)).astype(np.float32)
    return X, T


def test_param_count():
    assert N.lib().bmm_mlp_param_count() == O.N_PARAMS


def test_forward_matches_oracle(net):
    p = _params(net)
    assert np.all(p[O.B1:O.W2] == 0) and np.abs(p[O.W1:O.B1]).max() < 0.1
    # non-zero biases exercise the epilogue
    p[O.B1:O.W2] = np.linspace(-0.2, 0.2, 256)
    p[O.B3:] = np.linspace(0.1, -0.1, 256)
    N.check(N.lib().bmm_mlp_set_params(net, N.f32p(p)))
    X, _ = _inputs(257, 1)
    logits = np.zeros((257, 256), np.float32)
    N.check(N.lib().bmm_mlp_forward(net, N.f32p(X), 257, N.f32p(logits)))
    want = O.forward(p, X)[-1]
    assert np.allclose(logits, want, rtol=2e-3, atol=2e-3 * np.abs(want).max())


@pytest.mark.parametrize("rows", [1, 64, 200, 1000])
def test_gradients_match_oracle(net, rows):
    p = _params(net)
    X, T = _inputs(rows, rows)
    g = np.zeros(O.N_PARAMS, np.float32)
    loss = C.c_float(0)
    N.check(N.lib().bmm_mlp_grads(net, N.f32p(X), N.f32p(T), rows, N.f32p(g), C.byref(loss)))
    want_loss, want = O.loss_and_grads(p, X, T)
    assert abs(loss.value - want_loss) <= 1e-3 * max(1.0, abs(want_loss))
    for name, a, b in [("W1", O.W1, O.B1), ("b1", O.B1, O.W2), ("W2", O.W2, O.B2),
                       ("b2", O.B2, O.W3), ("W3", O.W3, O.B3), ("b3", O.B3, O.N_PARAMS)]:
        err = np.linalg.norm(g[a:b] - want[a:b]) / max(np.linalg.norm(want[a:b]), 1e-12)
        assert err < 1e-2, (name, err)


def test_adam_training_follows_oracle_and_learns(net):
    p = _params(net).astype(np.float64)
    X, T = _inputs(512, 9)
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    losses = []
    for step in range(1, 6):
        loss, g = O.loss_and_grads(p.astype(np.float32), X, T)
        losses.append(loss)
        p, m, v = O.adam(p, g, m, v, step)
    got_loss = C.c_float(0)
    N.check(N.lib().bmm_mlp_train(net, N.f32p(X), N.f32p(T), 512, 5, C.byref(got_loss)))
    assert abs(got_loss.value - losses[-1]) < 1e-2 * abs(losses[-1])
    got = _params(net)
    # Adam normalises every coordinate's step, so FP32-order differences in
    # near-zero gradients become full-size steps: compare with that slack
    rel = np.linalg.norm(got - p) / np.linalg.norm(p)
    assert rel < 5e-3
    # and it learns: 200 more steps cut the loss well below the start
    N.check(N.lib().bmm_mlp_train(net, N.f32p(X), N.f32p(T), 512, 200, C.byref(got_loss)))
    assert got_loss.value < 0.8 * losses[0]


def test_device_entry_points_match_host_ones():
    # bmm_mlp_create_on_stream + bmm_mlp_forward_dev / bmm_mlp_train_dev run the
    # same kernels as the host-pointer entry points, on the caller's stream:
    # same logits and, after the same training steps, the same parameters
    import torch

    X, T = _inputs(700, 9)
    stream = torch.cuda.Stream()
    L = N.lib()
    a, b = C.c_void_p(), C.c_void_p()
    N.check(L.bmm_mlp_create(5, 1e-3, C.byref(a)))
    N.check(L.bmm_mlp_create_on_stream(5, 1e-3, stream.cuda_stream, C.byref(b)))
    try:
        dx, dt = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
        dl = torch.empty((700, 256), device="cuda")
        torch.cuda.synchronize()
        want = np.zeros((700, 256), np.float32)
        N.check(L.bmm_mlp_forward(a, N.f32p(X), 700, N.f32p(want)))
        N.check(L.bmm_mlp_forward_dev(b, dx.data_ptr(), 700, dl.data_ptr()))
        stream.synchronize()
        assert np.array_equal(dl.cpu().numpy(), want)
        loss = np.zeros(1, np.float32)
        N.check(L.bmm_mlp_train(a, N.f32p(X), N.f32p(T), 700, 3, N.f32p(loss)))
        N.check(L.bmm_mlp_train_dev(b, dx.data_ptr(), dt.data_ptr(), 700, 3))
        stream.synchronize()
        assert np.array_equal(_params(a), _params(b))
        with pytest.raises(ValueError, match="null stream"):
            h = C.c_void_p()
            N.check(L.bmm_mlp_create_on_stream(5, 1e-3, None, C.byref(h)))
    finally:
        L.bmm_mlp_destroy(a)
        L.bmm_mlp_destroy(b)


@pytest.mark.parametrize("rows", [16384, 1000, 77])
def test_tma_forward_matches_thread_staging(rows):
    """BF16 features through the forward pass: the TMA-fed GEMMs (128-byte
    swizzled tiles, 4-stage ring) give exactly what the thread-staged GEMMs
    give, including row counts that leave a partial 128-row tile, and match
    the oracle's forward pass."""
    import torch

    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev).manual_seed(rows)
    x = torch.rand((rows, 512), generator=g, device=dev).to(torch.bfloat16)
    h = C.c_void_p()
    L = N.lib()
    N.check(L.bmm_mlp_create(11, 1e-3, C.byref(h)))
    try:
        outs = {}
        for tma in (1, 0):
            N.check(L.bmm_mlp_tune(tma))
            logits = torch.empty((rows, 256), device=dev)
            N.check(L.bmm_mlp_forward_bf16_dev(h, x.data_ptr(), rows, logits.data_ptr()))
            torch.cuda.synchronize()
            outs[tma] = logits.cpu().numpy()
        assert np.array_equal(outs[0], outs[1])
        params = np.zeros(N.lib().bmm_mlp_param_count(), np.float32)
        N.check(L.bmm_mlp_get_params(h, N.f32p(params)))
        xf = x.float().cpu().numpy()
        want = O.forward(params, xf)[-1]
        assert np.allclose(outs[1], want, rtol=2e-3, atol=2e-3 * np.abs(want).max())
    finally:
        N.check(L.bmm_mlp_tune(1))
        N.check(L.bmm_mlp_destroy(h))
