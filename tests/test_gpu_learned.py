"""The learned tail extrapolator: kernels and gradients against the numpy
oracle, and what the trained network gains over plain truncation."""

import math

import numpy as np
import pytest

from tbplas_b200 import _native as nat

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def _bf16_exact(rng, shape):
    from oracle.learned_oracle import bf16
    return bf16(rng.standard_normal(shape)).astype(np.float32)


@pytest.mark.parametrize("M,N,K", [(256, 128, 64), (200, 130, 72), (7, 300, 1280), (129, 3584, 16)])
def test_gemm_tn_matches_numpy(M, N, K):
    torch = _torch()
    lib = nat.load_library()
    rng = np.random.default_rng(M + N + K)
    a = _bf16_exact(rng, (M, K))
    b = _bf16_exact(rng, (N, K))
    c0 = rng.standard_normal((M, N)).astype(np.float32)
    A = torch.tensor(a, device="cuda").to(torch.bfloat16)
    B = torch.tensor(b, device="cuda").to(torch.bfloat16)
    C = torch.tensor(c0, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    assert lib.tbpm_nn_gemm_tn(A.data_ptr(), K, B.data_ptr(), K, C.data_ptr(), N, M, N, K,
                               0.5, 2.0, s) == 0
    ref = 0.5 * (a.astype(np.float64) @ b.astype(np.float64).T) + 2.0 * c0
    got = C.cpu().numpy()
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-5


def test_gemm_rejects_misaligned_shapes():
    torch = _torch()
    lib = nat.load_library()
    A = torch.zeros((16, 12), dtype=torch.bfloat16, device="cuda")
    C = torch.zeros((16, 16), dtype=torch.float32, device="cuda")
    assert lib.tbpm_nn_gemm_tn(A.data_ptr(), 12, A.data_ptr(), 12, C.data_ptr(), 16, 16, 16, 12,
                               1.0, 0.0, 0) == nat.TBPM_ERR_ARG


def test_im2col_col2im_are_adjoint():
    torch = _torch()
    lib = nat.load_library()
    from oracle.learned_oracle import im2col, col2im, bf16
    rng = np.random.default_rng(3)
    B, L, C, k, s, p = 3, 37, 8, 5, 2, 2
    Lout = (L + 2 * p - k) // s + 1
    x = bf16(rng.standard_normal((B, L, C)))
    X = torch.tensor(x, device="cuda").to(torch.bfloat16)
    Xc = torch.empty((B * Lout, k * C), dtype=torch.bfloat16, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    assert lib.tbpm_nn_im2col(X.data_ptr(), B, L, C, k, s, p, Lout, Xc.data_ptr(), st) == 0
    assert np.array_equal(Xc.float().cpu().numpy(), im2col(x, k, s, p, Lout))
    y = rng.standard_normal((B * Lout, k * C)).astype(np.float32)
    Y = torch.tensor(y, device="cuda")
    dX = torch.empty((B, L, C), dtype=torch.float32, device="cuda")
    assert lib.tbpm_nn_col2im(Y.data_ptr(), B, L, C, k, s, p, Lout, dX.data_ptr(), st) == 0
    assert np.allclose(dX.cpu().numpy(), col2im(y.astype(np.float64), B, L, C, k, s, p, Lout),
                       rtol=1e-5, atol=1e-5)


def test_network_gradients_match_oracle():
    from tbplas_b200.learned import TailNet
    from oracle.learned_oracle import forward_backward
    torch = _torch()
    net = TailNet(n_in=64, n_out=48, width=32, seed=5)
    rng = np.random.default_rng(11)
    B = 16
    x = rng.standard_normal((B, 64, 2)).astype(np.float32) * 0.3
    y = rng.standard_normal((B, 48, 2)).astype(np.float32) * 0.1
    pred = net.forward(x, keep=True)
    target = torch.tensor(y.reshape(B, -1), device="cuda")
    loss, grad = net.loss_and_grad(pred, target)
    net.backward(grad)
    params = [p["w"].cpu().numpy().astype(np.float64) for p in net.params]
    xp = np.zeros((B, 64, net.c_in))
    xp[:, :, :2] = x * net.in_scale
    ref_loss, ref_out, ref_grads = forward_backward(params, net.convs, net.kernel, net.F, xp,
                                                    y.reshape(B, -1).astype(np.float64))
    out = pred.cpu().numpy()
    assert np.max(np.abs(out - ref_out)) / np.max(np.abs(ref_out)) < 5e-3
    assert abs(float(loss.item()) - ref_loss) / ref_loss < 5e-3
    for p, g in zip(net.params, ref_grads):
        got = p["g"].cpu().numpy()
        rel = np.linalg.norm(got - g) / max(np.linalg.norm(g), 1e-30)
        assert rel < 1e-2, rel


def test_training_reduces_loss():
    from tbplas_b200.learned import TailNet
    rng = np.random.default_rng(0)
    n, n_in, n_out = 256, 64, 48
    t = np.arange(1, n_in + n_out + 1)
    decay = rng.uniform(0.005, 0.05, n)[:, None]
    freq = rng.uniform(0.05, 0.4, n)[:, None]
    c = np.exp(-decay * t) * np.exp(-1j * freq * t)
    x = np.stack([c[:, :n_in].real, c[:, :n_in].imag], -1).astype(np.float32)
    y = np.stack([c[:, n_in:].real, c[:, n_in:].imag], -1).astype(np.float32)
    net = TailNet(n_in=n_in, n_out=n_out, width=32, seed=1)
    net.fit_scales(x, y)
    before = net.mse(x, y)
    net.train(x, y, epochs=60, batch=32, lr=2e-3)
    after = net.mse(x, y)
    assert after < 0.05 * before


def test_learned_tail_beats_truncation_when_the_tail_is_deterministic():
    """Weakly disordered graphene averaged over many states: C(t) beyond the
    short window still carries the DOS fine structure.  A network trained on
    GPU-generated curves of other realisations must give a DOS closer to the
    full-length propagation than the DOS of the short window alone."""
    import math
    import tbplas_b200 as tb
    from tbplas_b200.fortran import f2py
    from tbplas_b200.learned import TailNet, curves_to_xy, dos_l1, extend
    from conftest import bessel_series
    n_in, tnr, ns = 64, 512, 64
    rng = np.random.default_rng(5)

    def batch(n, seed0):
        samples = [tb.make_graphene_sample(48, 48, disorder=float(rng.uniform(0, 0.2)),
                                           rescale=10.0, seed=seed0 + i) for i in range(n)]
        p = tb.pack_samples(samples)
        f2py.set_backend(precision="fp32")
        try:
            return f2py.tbpm_dos_segmented(bessel_series(math.pi), p.indptr, p.indices, p.data,
                                           p.offsets, ns, seed0, tnr)
        finally:
            f2py.set_backend(precision="fp64")

    train = batch(96, 100)
    test = batch(16, 900)
    x, y = curves_to_xy(train, n_in, tnr - n_in)
    net = TailNet(n_in=n_in, n_out=tnr - n_in, width=64, seed=3)
    net.fit_scales(x, y)
    net.train(x[16:], y[16:], epochs=300, batch=16, lr=1e-3, weight_decay=1e-3,
              x_val=x[:16], y_val=y[:16], patience=60)
    xs, _ = curves_to_xy(test, n_in, tnr - n_in)
    learned = extend(test[:, :n_in + 1], net.predict(xs))
    l1_learned = np.mean([dos_l1(learned[k], test[k], 20.0) for k in range(16)])
    l1_trunc = np.mean([dos_l1(test[k, :n_in + 1], test[k], 20.0) for k in range(16)])
    assert l1_learned < 0.8 * l1_trunc, (l1_learned, l1_trunc)
