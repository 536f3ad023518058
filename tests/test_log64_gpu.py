"""The FP64 integrands' logarithm (ccoil_eval_log64) against the host's double
logarithm: within 1 ulp, and equal to it in more than 99 % of cases, over the
whole exponent range, near 1 (where the vector potential's log of a ratio of
nearly equal sums lands for far points) and on the reduction interval's edges.
The refinement pass's reciprocal square root and division (ccoil_eval_rsqrt64,
ccoil_eval_div64) against the host's extended precision rounded to double."""
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


def test_rsqrt64_within_one_ulp(ccoil):
    import torch
    rng = np.random.default_rng(43)
    x = np.concatenate([
        np.exp(rng.uniform(np.log(1e-36), np.log(1e36), 200000)),   # the unchecked form's range
        np.ldexp(1.0, rng.integers(-110, 110, 20000)) * (1.0 + rng.uniform(-1e-12, 1e-12, 20000)),
        rng.uniform(1e-4, 10.0, 100000),                              # squared distances of the workloads
    ])
    xd = torch.from_numpy(x).cuda()
    out = torch.empty_like(xd)
    assert ccoil.lib().ccoil_eval_rsqrt64(xd.data_ptr(), out.data_ptr(), len(x), None) == 0
    ref = _extended_ref(1 / np.sqrt(x.astype(np.longdouble)))
    e = ulp_error(out.cpu().numpy(), ref)
    assert e.max() <= 1.0, (e.max(), x[np.argmax(e)])


def test_div64_within_one_ulp(ccoil):
    import torch
    rng = np.random.default_rng(47)
    n = 200000
    den = np.exp(rng.uniform(np.log(1e-36), np.log(1e36), n))
    num = np.exp(rng.uniform(np.log(1e-30), np.log(1e30), n)) * rng.choice([-1.0, 1.0], n)
    near = 1.0 + rng.uniform(-1e-6, 1e-6, 50000)                     # ratios of nearly equal products
    den = np.concatenate([den, near])
    num = np.concatenate([num, near * (1.0 + rng.uniform(-1e-9, 1e-9, 50000))])
    nd, dd = torch.from_numpy(num).cuda(), torch.from_numpy(den).cuda()
    out = torch.empty_like(nd)
    assert ccoil.lib().ccoil_eval_div64(nd.data_ptr(), dd.data_ptr(), out.data_ptr(), len(num), None) == 0
    ref = _extended_ref(num.astype(np.longdouble) / den.astype(np.longdouble))
    e = ulp_error(out.cpu().numpy(), ref)
    assert e.max() <= 1.0, (e.max(), num[np.argmax(e)], den[np.argmax(e)])
    assert np.mean(e > 0.5) < 0.01, np.mean(e > 0.5)  # nearly always correctly rounded
