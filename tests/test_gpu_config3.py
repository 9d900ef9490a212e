"""Config 3 as specified: CoeffToSlot and SlotToCoeff on 8 real encryptions of seeded uniform
complex slots with |z| <= 1, through the whole plans, against the reference.

The reference's walsh15 bootstrapping context (its keys and secret) supplies the rotation keys;
the device uses the plans it generates itself (wg_dft_plan_create, the reference's literals),
the reference its own plans.  8 slot vectors are encoded and encrypted under the reference
context's secret on the device (wg_encode_slots_device, wg_encrypt_symmetric with a drawn mask
and noise), CoeffToSlot at the top level (12) and SlotToCoeff at its entry level (1) run as one
batch of 8 on the device and ciphertext by ciphertext through the reference's QP stage
evaluator (ckks_apply_linear_transform_owned_stage_qp, stage after stage as
ckks_apply_linear_transform_plan does, src/ckks/operations/bootstrap/ckks_linear_transform.cpp:
1409-1427).  Every output residue must be the reference's, and the decoded FP64 slots (the
reference's decryptor) then agree exactly; their magnitude is reported."""
import numpy as np
import pytest

from test_dft_plan import _literals

pytestmark = pytest.mark.gpu

BATCH = 8


@pytest.fixture(scope="module")
def walsh15(ref_mod):
    return ref_mod.RefPlans(bootstrap_keys=True)


@pytest.mark.parametrize("which", ["c2s", "s2c"])
def test_plan_on_encrypted_slots_matches_reference(wg, walsh15, which):
    import torch

    R = walsh15
    N, half = R.N, R.N // 2
    info = R.bts_info()
    code, lit = _literals(wg, R)[which]
    level = info["depth"] if which == "c2s" else info["s2c_depth"]
    ctx = wg.Context(N, R.q, R.p, R.dnum)
    for r in R.rotations():
        k, parts, kl = R.key(int(r))
        ctx.set_key(wg.WG_KEY_ROTATION, k, rotation=int(r), parts=parts, key_level=kl)
    stages = ctx.dft_plan(lit)
    assert len(stages) == R.stages(code)

    rng = np.random.default_rng(33 if which == "c2s" else 34)
    rad = np.sqrt(rng.random((BATCH, half)))
    ang = 2 * np.pi * rng.random((BATCH, half))
    z = rad * np.exp(1j * ang)  # uniform on the unit disc
    n = (level + 1) * N
    pts = [torch.empty(n, dtype=torch.int64, device="cuda") for _ in range(BATCH)]
    ctx.encode_slots_device(level + 1, R.scale, z.real, z.imag, pts, eval_form=True)
    full = (info["depth"] + 1) * N
    cts = [(torch.zeros(full, dtype=torch.int64, device="cuda"), torch.zeros(full, dtype=torch.int64, device="cuda"))
           for _ in range(BATCH)]
    ctx.encrypt_symmetric(level, pts, R.secret_coeffs(), cts, seed=77)
    torch.cuda.synchronize()
    inputs = [(wg.to_host(b)[:n], wg.to_host(a)[:n]) for b, a in cts]

    lv = level
    for st in stages:
        st.apply([c[0] for c in cts], [c[1] for c in cts])
        lv = st.info()["level"] - (1 if st.info()["rescale"] else 0)
    torch.cuda.synchronize()

    worst = 0.0
    for k, (b, a) in enumerate(inputs):
        rl = level
        for s in range(R.stages(code)):
            b, a, rl = R.apply_stage(code, s, rl, b, a)
        assert rl == lv
        m = (rl + 1) * N
        gb, ga = wg.to_host(cts[k][0])[:m], wg.to_host(cts[k][1])[:m]
        assert (gb == b[:m]).all() and (ga == a[:m]).all(), (which, k, int((gb != b[:m]).sum()))
        dec_dev = R.decrypt(rl, R.scale, gb, ga)
        dec_ref = R.decrypt(rl, R.scale, b[:m], a[:m])
        assert np.array_equal(dec_dev, dec_ref)
        worst = max(worst, float(np.abs(dec_dev).max()))
    assert np.isfinite(worst)
    print(f"{which}: {BATCH} encryptions of |z| <= 1 through {len(stages)} stages, residues equal to the reference's; "
          f"decoded |slot| up to {worst:.3g} at the parameter scale")
    for st in stages:
        st.close()
