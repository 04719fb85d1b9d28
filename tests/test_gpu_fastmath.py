"""The fast build's reciprocal (bnz_fastmath.cuh), which replaces the van Leer
limiter's division there, checked against the IEEE quotient (numpy's 1/x,
correctly rounded, as CUDA's double division is): within 2 ulp for every x
whose reciprocal is a normal number, across the exponent range and the
mantissa patterns near powers of two."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ulp_err(y, r):
    return np.abs(y - r) / np.spacing(np.abs(r))


def test_fast_rcp_within_two_ulp():
    import torch
    from bonzo_b200._lib import fast_rcp
    rng = np.random.default_rng(7)
    n = 1 << 20
    mant = rng.uniform(1.0, 2.0, n)
    expo = rng.integers(-1000, 1000, n)
    x = np.ldexp(mant, expo) * np.where(rng.random(n) < 0.5, -1.0, 1.0)
    edge = np.concatenate([np.ldexp(1.0, np.arange(-1000, 1000)),
                           np.nextafter(np.ldexp(1.0, np.arange(-1000, 1000)), 0.0),
                           np.nextafter(np.ldexp(1.0, np.arange(-1000, 1000)), np.inf),
                           [1.0, 3.0, 1.0 / 3.0, 0.1, 7.0e-20, 2.5e19]])
    x = np.concatenate([x, edge, -edge])
    y = fast_rcp(torch.from_numpy(x).cuda()).cpu().numpy()
    r = 1.0 / x
    err = _ulp_err(y, r)
    assert np.all(np.isfinite(y))
    assert err.max() <= 2.0, (x[np.argmax(err)], err.max())
    # the limiter's use: 2ab / (a + b) for same-signed slopes
    a = rng.standard_normal(n) * 10.0 ** rng.integers(-12, 3, n)
    b = np.abs(rng.standard_normal(n)) * np.sign(a) * 10.0 ** rng.integers(-12, 3, n)
    s = a + b
    lim = (2.0 * a * b) * fast_rcp(torch.from_numpy(s).cuda()).cpu().numpy()
    ref = 2.0 * a * b / s
    assert (np.abs(lim - ref) <= 4 * np.spacing(np.abs(ref))).all()


def test_fast_rcp_rejects_bad_arguments():
    from bonzo_b200._lib import BNZ_ERR_ARG, load
    L = load()
    assert L.bnz_fast_rcp(None, None, -1, None) == BNZ_ERR_ARG
    assert L.bnz_fast_rcp(None, None, 4, None) == BNZ_ERR_ARG
    assert L.bnz_fast_rcp(None, None, 0, None) == 0
