"""The FP64 integrands' logarithm (ccoil_eval_log64) against the host's double
logarithm: within 1 ulp, and equal to it in more than 99 % of cases, over the
whole exponent range, near 1 (where the vector potential's log of a ratio of
nearly equal sums lands for far points) and on the reduction interval's edges.
The refinement pass's reciprocal square root, square root, division and
logarithm of a ratio (ccoil_eval_fp64_op) against the host's extended precision
rounded to double."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def ulp_error(got, ref):
    return np.abs(got - ref) / np.spacing(np.abs(ref))


def test_log64_within_one_ulp(ccoil):
    import torch
    rng = np.random.default_rng(41)
    s = np.sqrt(0.5)
    x = np.concatenate([
        np.exp(rng.uniform(-700.0, 700.0, 200000)),                # whole range
        1.0 + rng.uniform(-1e-3, 1e-3, 100000),                    # near 1
        1.0 + rng.uniform(-1e-12, 1e-12, 20000),
        rng.uniform(0.25, 4.0, 100000),
        np.nextafter(s, 0.0) * (1.0 + rng.uniform(-1e-9, 1e-9, 10000)),  # reduction edges
        np.nextafter(np.sqrt(2.0), 3.0) * (1.0 + rng.uniform(-1e-9, 1e-9, 10000)),
    ])
    x = x[x != 1.0]
    xd = torch.from_numpy(x).cuda()
    out = torch.empty_like(xd)
    assert ccoil.lib().ccoil_eval_log64(xd.data_ptr(), out.data_ptr(), len(x), None) == 0
    e = ulp_error(out.cpu().numpy(), np.log(x))
    assert e.max() <= 1.0, (e.max(), x[np.argmax(e)])
    assert np.mean(e > 0.5) < 0.01, np.mean(e > 0.5)  # nearly always correctly rounded


def _extended_ref(v):
    """Round an extended-precision host result to double (needs a long double
    wider than double, as on x86-64)."""
    assert np.finfo(np.longdouble).nmant > 52
    return v.astype(np.float64)


def _fp64_op(ccoil, op, a, b=None):
    import torch
    ad = torch.from_numpy(a).cuda()
    bd = torch.from_numpy(b).cuda() if b is not None else None
    out = torch.empty_like(ad)
    assert ccoil.lib().ccoil_eval_fp64_op(op, ad.data_ptr(), bd.data_ptr() if bd is not None else None,
                                          out.data_ptr(), len(a), None) == 0
    return out.cpu().numpy()


def _roots_args(seed):
    rng = np.random.default_rng(seed)
    return np.concatenate([
        np.exp(rng.uniform(np.log(1e-36), np.log(1e36), 200000)),   # the unchecked forms' range
        np.ldexp(1.0, rng.integers(-110, 110, 20000)) * (1.0 + rng.uniform(-1e-12, 1e-12, 20000)),
        rng.uniform(1e-4, 10.0, 100000),                              # squared distances of the workloads
    ])


def test_rsqrt64_within_one_ulp(ccoil):
    x = _roots_args(43)
    e = ulp_error(_fp64_op(ccoil, 0, x), _extended_ref(1 / np.sqrt(x.astype(np.longdouble))))
    assert e.max() <= 1.0, (e.max(), x[np.argmax(e)])


def test_sqrt64_within_one_ulp(ccoil):
    x = _roots_args(44)
    e = ulp_error(_fp64_op(ccoil, 1, x), _extended_ref(np.sqrt(x.astype(np.longdouble))))
    assert e.max() <= 1.0, (e.max(), x[np.argmax(e)])


def _ratio_args(seed):
    rng = np.random.default_rng(seed)
    n = 200000
    den = np.exp(rng.uniform(np.log(1e-36), np.log(1e36), n))
    num = np.exp(rng.uniform(np.log(1e-30), np.log(1e30), n))
    near = 1.0 + rng.uniform(-1e-6, 1e-6, 50000)                     # ratios of nearly equal products
    den = np.concatenate([den, near, np.sqrt(2.0) * near])           # and at the fold's edges
    num = np.concatenate([num, near * (1.0 + rng.uniform(-1e-9, 1e-9, 50000)), near])
    return num, den


def test_div64_within_one_ulp(ccoil):
    num, den = _ratio_args(47)
    num = num * np.random.default_rng(48).choice([-1.0, 1.0], len(num))
    ref = _extended_ref(num.astype(np.longdouble) / den.astype(np.longdouble))
    e = ulp_error(_fp64_op(ccoil, 2, num, den), ref)
    assert e.max() <= 1.0, (e.max(), num[np.argmax(e)], den[np.argmax(e)])
    assert np.mean(e > 0.5) < 0.01, np.mean(e > 0.5)  # nearly always correctly rounded


def test_log_ratio64_within_four_ulp(ccoil):
    """log(n / d) without the rounded quotient: within a few ulp of the true
    logarithm even where n / d is within 1e-9 of 1 (where log64 of a rounded
    quotient would be off by up to 1e-7 relative)."""
    num, den = _ratio_args(49)
    # within a factor 2 of 1: log1p of (n - d) / d, n - d exact (a rounded
    # extended quotient alone would be off by ~1e-19 absolute there, 1e5 ulp of
    # a logarithm of 1e-9); elsewhere the extended logarithm of the quotient
    nl, dl = num.astype(np.longdouble), den.astype(np.longdouble)
    q = nl / dl
    near = (q > 0.5) & (q < 2.0)
    ref = _extended_ref(np.where(near, np.log1p(np.where(near, (nl - dl) / dl, 0.0)), np.log(q)))
    e = ulp_error(_fp64_op(ccoil, 3, num, den), ref)
    assert e.max() <= 4.0, (e.max(), num[np.argmax(e)], den[np.argmax(e)])
