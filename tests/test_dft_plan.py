"""The library's bootstrapping DFT plan generator (host part, no device) against the reference's
own walsh15 plans (ckks_generate_bootstrap_dft_plan, src/ckks/operations/bootstrap/
ckks_bootstrap_dft.cpp:961-1079, built by the reference's context from its AESWalsh15
parameters): SlotToCoeff at the parameter scale and at twice it, and CoeffToSlot.

Per stage: level, rescale flag, baby-step count and the diagonal index set must be the
reference's; and the generated diagonals, rotated by their giant-step offset and encoded over
the stage's QP basis with the library's host encoder (the reference's FP64 encoder steps),
transformed by the oracle's NTT and put in Montgomery form, must give the reference's stored
QP plaintext words (compared modulo q: the device test compares the device-encoded words
exactly)."""
import numpy as np
import pytest


def _literals(wg, R):
    info = R.bts_info()
    q0, scale = float(R.q[0]), info["scale"]
    K = wg.evalmod_k_bound(1 << 15, 32, -16.0)
    s2c = lambda ratio: wg.DftLiteral.make(False, info["s2c_depth"], (q0 * 0.5) / (scale * ratio),
                                           scale_groups=[[18, 20, 23]], active_slots=16384, log_bsgs_ratio=1)
    # binary_c2s_transform_scale (ckks_evalmod_scale_plan.hpp:21-45): 2^(38 - 36) scale / q0 / K
    c2s_scale = np.ldexp(scale, 38 - 36) / q0 / K
    c2s = wg.DftLiteral.make(True, info["depth"], c2s_scale, scale_groups=[[25, 25], [25, 25]], active_slots=16384,
                             log_bsgs_ratio=1)
    return {"s2c": (0, s2c(1)), "s2c_x2": (None, s2c(2)), "c2s": (1, c2s)}


@pytest.fixture(scope="module")
def walsh15_plans(ref_mod):
    return ref_mod.RefPlans(bootstrap_keys=True)


def _montgomery(x, q):
    r = (1 << 64) % int(q)
    return (x.astype(object) * r) % int(q)


@pytest.mark.parametrize("which", ["s2c", "c2s", "s2c_x2"])
def test_plan_matches_reference(wg, oracle_mod, walsh15_plans, which):
    R = walsh15_plans
    N, K = R.N, len(R.p)
    code, lit = _literals(wg, R)[which]
    if code is None:
        code = R.build_scaled_s2c(2)
    nst = R.stages(code)
    o = oracle_mod.OracleCtx(N, R.q, R.p, R.dnum)
    mine0 = wg.dft_plan_describe(N, R.q, lit, 0)
    assert mine0["stages"] == nst
    full = N // 2
    for k in range(nst):
        ref = R.stage(code, k)
        mine = wg.dft_plan_describe(N, R.q, lit, k, diagonals=True)
        assert mine["nterms"] == ref["nterms"], k
        assert mine["baby"] == ref["baby"], k
        assert mine["rescale"] == ref["rescale"], k
        assert mine["level"] + 1 + K == ref["qp_limbs"], k
        assert (mine["indices"] == ref["indices"]).all(), k
        T = ref["qp_limbs"]
        moduli = np.concatenate([R.q[: mine["level"] + 1], R.p])
        ref_d = ref["diagonals"].reshape(ref["nterms"], T, N)
        terms = sorted({0, ref["nterms"] // 2, ref["nterms"] - 1})
        for t in terms:
            d = mine["diagonals"][t]
            rot = (int(mine["indices"][t]) // mine["baby"]) * mine["baby"]
            src = ((np.arange(full) + full - rot) & (full - 1)) % d.size
            v = d[src]
            coeffs = wg.encode_slots(N, v.real, v.imag, mine["plaintext_scale"], moduli).reshape(T, N)
            L = mine["level"] + 1
            evq = o.ntt(coeffs[:L].reshape(-1)).reshape(L, N)
            evp = o.ntt(coeffs[L:].reshape(-1), which=1).reshape(K, N)
            ev = np.concatenate([evq, evp])
            for limb in range(T):
                m = int(moduli[limb])
                got = _montgomery(ev[limb], m)
                want = ref_d[t, limb].astype(object) % m
                assert (got == want).all(), (which, k, t, limb, int((got != want).sum()))
