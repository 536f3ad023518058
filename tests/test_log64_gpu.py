"""The FP64 integrands' logarithm (ccoil_eval_log64) against the host's double
logarithm: within 1 ulp, and equal to it in more than 99 % of cases, over the
whole exponent range, near 1 (where the vector potential's log of a ratio of
nearly equal sums lands for far points) and on the reduction interval's edges."""
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
