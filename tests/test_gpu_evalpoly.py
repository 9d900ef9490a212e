"""Chebyshev polynomial evaluation on the device against the reference's
ckks_evalchebyshev_preconditioned (compiled from its own sources) on the walsh15 chain: same
input residues, coefficients and relinearisation key; output residues, level and scale must be
identical.  Shapes cover mixed, odd-only and even-only series, degree 0, and the degree-100
even series of the walsh15 EvalMod step (levels 10 -> 3), over a batch of ciphertexts."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def plans(ref_mod):
    return ref_mod.RefPlans()


@pytest.fixture(scope="module")
def gpu_ctx(wg, plans):
    ctx = wg.Context(plans.N, plans.q, plans.p, plans.dnum)
    key, parts, kl = plans.key(0, kind=2)
    ctx.set_key(wg.WG_KEY_RELIN, key, parts=parts, key_level=kl)
    return ctx


def _series(kind, degree, rng):
    c = rng.uniform(-1.0, 1.0, degree + 1) / (1.0 + np.arange(degree + 1)) ** 0.5
    if kind == "odd":
        c[0::2] = 0.0
    elif kind == "even":
        c[1::2] = 0.0
    return c


CASES = [("mixed", 7, 10), ("mixed", 23, 10), ("odd", 15, 9), ("even", 30, 10), ("even", 100, 10), ("mixed", 0, 4),
         ("mixed", 1, 4), ("mixed", 2, 5)]


@pytest.mark.parametrize("kind,degree,level", CASES)
def test_evalchebyshev_matches_reference(wg, plans, gpu_ctx, kind, degree, level):
    import torch

    N = plans.N
    rng = np.random.default_rng(degree * 7 + level)
    coeffs = _series(kind, degree, rng)
    if degree == 0:
        coeffs = np.array([0.375])
    qc = np.repeat(plans.q[: level + 1], N)
    count = 2
    ins = [((rng.integers(0, 1 << 62, (level + 1) * N, dtype=np.uint64) % qc).astype(np.uint64),
            (rng.integers(0, 1 << 62, (level + 1) * N, dtype=np.uint64) % qc).astype(np.uint64)) for _ in range(count)]
    db = [wg.to_device(b) for b, _ in ins]
    da = [wg.to_device(a) for _, a in ins]
    ob = [torch.empty((level + 1) * N, dtype=torch.int64, device="cuda") for _ in range(count)]
    oa = [torch.empty((level + 1) * N, dtype=torch.int64, device="cuda") for _ in range(count)]
    lvl, sc = gpu_ctx.evalchebyshev(level, plans.scale, coeffs, db, da, ob, oa, default_scale=plans.scale)
    torch.cuda.synchronize()
    for k, (b, a) in enumerate(ins):
        rb, ra, rl, rs = plans.evalchebyshev(level, plans.scale, coeffs, b, a)
        assert (lvl, sc) == (rl, rs)
        n = (rl + 1) * N
        gb, ga = wg.to_host(ob[k])[:n], wg.to_host(oa[k])[:n]
        assert (gb == rb).all(), (kind, degree, k, int((gb != rb).sum()))
        assert (ga == ra).all(), (kind, degree, k, int((ga != ra).sum()))
        # the inputs are read only
        assert (wg.to_host(db[k]) == b).all() and (wg.to_host(da[k]) == a).all()


def test_evalchebyshev_level_too_small(wg, plans, gpu_ctx):
    import torch

    N = plans.N
    t = torch.zeros(2 * N, dtype=torch.int64, device="cuda")
    with pytest.raises(wg.InvalidArgument):
        gpu_ctx.evalchebyshev(1, plans.scale, np.ones(17), [t], [t.clone()], [t.clone()], [t.clone()],
                              default_scale=plans.scale)
