"""The hot path's division and square root (p2r_math_check) against correctly rounded
results: the default build refines the hardware reciprocal / reciprocal square root by one
Newton-Raphson step and must stay within 2 ulp over the argument ranges the path sees (the
per-step chained-filter accuracy it buys is covered by the parity tests)."""
import numpy as np
import pytest

BOUND_ULP = {"refined": 2, "ieee": 0, "fast": 3}


def _ulp_err(got: np.ndarray, exact: np.ndarray) -> np.ndarray:
    """|got - exact| in units of the float32 spacing at the correctly rounded result."""
    want = exact.astype(np.float32)
    return np.abs(got.astype(np.float64) - exact) / np.spacing(np.abs(want)).astype(np.float64)


@pytest.mark.gpu
def test_division_and_sqrt_within_bound():
    import torch
    import p2r_tests_b200 as p2r
    rng = np.random.default_rng(7)
    n = 1 << 22
    # magnitudes of the path's operands: 1/pT, radii, cosines, 2x2 determinants
    a = (np.exp(rng.uniform(np.log(1e-12), np.log(1e6), n)) * rng.choice([-1.0, 1.0], n)).astype(np.float32)
    b = (np.exp(rng.uniform(np.log(1e-6), np.log(1e6), n)) * rng.choice([-1.0, 1.0], n)).astype(np.float32)
    a_pos = np.abs(a)
    da, db = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    quot, _ = p2r.math_check(da, db)
    _, root = p2r.math_check(torch.from_numpy(a_pos).cuda(), db)
    torch.cuda.synchronize()
    q_exact = a.astype(np.float64) / b.astype(np.float64)
    r_exact = np.sqrt(a_pos.astype(np.float64))
    eq = _ulp_err(quot.cpu().numpy(), q_exact)
    er = _ulp_err(root.cpu().numpy(), r_exact)
    bound = BOUND_ULP[p2r.math_variant()]
    # the correctly rounded result itself is within 0.5 ulp of the exact one
    assert eq.max() <= bound + 0.5, f"division max {eq.max():.3f} ulp ({p2r.math_variant()})"
    assert er.max() <= bound + 0.5, f"sqrt max {er.max():.3f} ulp ({p2r.math_variant()})"
    print(f"{p2r.math_variant()}: div max {eq.max():.3f} mean {eq.mean():.3f} ulp; "
          f"sqrt max {er.max():.3f} mean {er.mean():.3f} ulp")


@pytest.mark.gpu
def test_sqrt_special_arguments():
    import torch
    import p2r_tests_b200 as p2r
    a = torch.tensor([0.0, -0.0, -1.0, float("inf"), float("nan"), 1e-30], device="cuda")
    _, root = p2r.math_check(a, torch.ones_like(a))
    r = root.cpu().numpy()
    # the path's square roots take sums of squares; a negative argument only has to give no root
    assert r[0] == 0.0 and not r[2] >= 0 and np.isnan(r[4])
    assert np.isinf(r[3]) or p2r.math_variant() != "ieee"
    assert abs(r[5] - 1e-15) / 1e-15 < 1e-5 or p2r.math_variant() == "fast"


def test_math_variant_is_declared():
    import p2r_tests_b200 as p2r
    assert p2r.math_variant() in BOUND_ULP
