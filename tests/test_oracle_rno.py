"""CPU test: the surrogate oracle's backward pass against central finite differences."""

from __future__ import annotations

import numpy as np
import pytest

from oracle.rno import IN_PAD, IN_REAL, OUT_PAD, window_forward_backward


def _params(rng, h):
    dims = [(h, IN_PAD), (h, h), (h, h), (OUT_PAD, h)]
    out = []
    for o, i in dims:
        W = rng.normal(0, 1.0 / np.sqrt(i), size=(o, i))
        if i == IN_PAD:
            W[:, IN_REAL:] = 0.0
        if o == OUT_PAD:
            W[12:] = 0.0
        out.append((W, rng.normal(0, 0.1, size=o) * (np.arange(o) < (12 if o == OUT_PAD else o))))
    return out


@pytest.mark.parametrize("with_skip", [False, True])
def test_oracle_window_gradients_match_finite_differences(with_skip: bool) -> None:
    rng = np.random.default_rng(0)
    h, T, B = 16, 4, 3
    params = _params(rng, h)
    strain, rate, target = (rng.normal(size=(T, B, 6)) for _ in range(3))
    coef = rng.uniform(0.05, 0.3, size=(T, B))
    z0 = rng.normal(size=(B, 6)) * 0.1
    skip = rng.normal(size=(6, 6)) * 0.5 if with_skip else None
    loss, grads, _, _ = window_forward_backward(params, strain, rate, target, coef, z0, skip=skip)
    eps = 1e-6
    for li, (W, b) in enumerate(params):
        for arr, g in ((W, grads[li][0]), (b, grads[li][1])):
            flat = arr.reshape(-1)
            idx = rng.choice(flat.size, size=min(8, flat.size), replace=False)
            for k in idx:
                if (li == 0 and arr is W and (k % IN_PAD) >= IN_REAL) or (li == 3 and arr is W and k // h >= 12):
                    continue
                old = flat[k]
                flat[k] = old + eps
                lp = window_forward_backward(params, strain, rate, target, coef, z0, skip=skip)[0]
                flat[k] = old - eps
                lm = window_forward_backward(params, strain, rate, target, coef, z0, skip=skip)[0]
                flat[k] = old
                fd = (lp - lm) / (2 * eps)
                assert abs(fd - g.reshape(-1)[k]) <= 1e-6 * max(abs(fd), 1e-3), (li, k, fd, g.reshape(-1)[k])
