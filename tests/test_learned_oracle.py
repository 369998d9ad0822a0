"""Pin the numpy oracle of the learned extrapolator (no GPU): with bfloat16
rounding switched off its analytic gradients equal central finite
differences of its loss."""

import numpy as np

import oracle.learned_oracle as lo


def _geometry(n_in, width, kernel, strides, c_in):
    convs, L, C = [], n_in, c_in
    for s in strides:
        Lout = (L + 2 * (kernel // 2) - kernel) // s + 1
        convs.append({"L": L, "C": C, "Lout": Lout, "Cout": width, "s": s, "p": kernel // 2})
        L, C = Lout, width
    return convs, L * C


def test_oracle_gradients_equal_finite_differences(monkeypatch):
    monkeypatch.setattr(lo, "bf16", lambda x: np.asarray(x, dtype=np.float64))
    rng = np.random.default_rng(0)
    n_in, width, kernel, c_in, O, B = 16, 4, 3, 2, 6, 3
    convs, F = _geometry(n_in, width, kernel, (2, 2, 2), c_in)
    params = []
    for cv in convs:
        params += [rng.standard_normal((cv["Cout"], kernel * cv["C"])) * 0.5,
                   rng.standard_normal(cv["Cout"]) * 0.1]
    params += [rng.standard_normal((O, F)) * 0.3, rng.standard_normal(O) * 0.1]
    x = rng.standard_normal((B, n_in, c_in))
    y = rng.standard_normal((B, O))
    loss, _, grads = lo.forward_backward(params, convs, kernel, F, x, y)
    h = 1e-6
    for pi, p in enumerate(params):
        flat = p.reshape(-1)
        for idx in rng.choice(flat.size, size=min(6, flat.size), replace=False):
            old = flat[idx]
            flat[idx] = old + h
            lp, _, _ = lo.forward_backward(params, convs, kernel, F, x, y)
            flat[idx] = old - h
            lm, _, _ = lo.forward_backward(params, convs, kernel, F, x, y)
            flat[idx] = old
            fd = (lp - lm) / (2 * h)
            assert abs(fd - grads[pi].reshape(-1)[idx]) < 1e-6 * max(1.0, abs(fd))


def test_bf16_rounding_is_round_to_nearest_even():
    # 1 + 2^-8 is halfway between bf16 neighbours 1 and 1 + 2^-7: rounds to even (1)
    assert lo.bf16(np.array([1.0 + 2.0 ** -8]))[0] == 1.0
    assert lo.bf16(np.array([1.0 + 3 * 2.0 ** -8]))[0] == 1.0 + 2.0 ** -6
    assert lo.bf16(np.array([-2.5]))[0] == -2.5
