"""The numpy restatement of the preconditioner network (the checker of the
device forward/backward): its analytic gradient against central finite
differences, BF16 rounding, and the parameter layout."""
import numpy as np


def test_oracle_gradient_matches_finite_differences():
    from oracle import precnet_oracle as P
    rng = np.random.default_rng(0)
    _, n = P.param_slices()
    w = rng.standard_normal(n) * 0.2
    x = rng.standard_normal((2, 2, 16, 16))
    dout = rng.standard_normal((2, 1, 16, 16))
    A = P.forward(w, x, round_weights=False)
    g = P.backward(w, A, dout, round_weights=False)
    for k in range(6):
        v = rng.standard_normal(n)
        eps = 1e-6
        lp = (P.forward(w + eps * v, x, False)[-1] * dout).sum()
        lm = (P.forward(w - eps * v, x, False)[-1] * dout).sum()
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g @ v) <= 1e-6 * max(1.0, abs(fd)), (fd, g @ v)


def test_bf16_rounding_and_layout():
    from oracle import precnet_oracle as P
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 65504.0, 1e-30], dtype=np.float32)
    r = P.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125
    assert np.all(np.abs(r - x) <= np.abs(x) * 2 ** -8)
    sl, n = P.param_slices()
    convs = [s for s in sl if s is not None]
    assert len(convs) == 12
    assert n == (16 * 2 * 9 + 16) + 10 * (16 * 16 * 9 + 16) + (16 * 9 + 1)
