"""CoeffToSlot / SlotToCoeff BSGS stages on the device against the reference itself.

The reference library compiled from its own sources (oracle/_ref, built where the sources
exist and shipped with the repository snapshot) builds the AESWalsh15 modulus chain with its
S2C and C2S plans and the rotation keys they need; its own QP stage evaluator
(ckks_apply_linear_transform_owned_stage_qp) gives the expected residues.  The device stage
gets the same diagonals and keys and runs a batch of ciphertexts at once; every residue must
match bit for bit.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def plans(ref_mod):
    return ref_mod.RefPlans()


@pytest.fixture(scope="module")
def gpu_ctx(wg, plans):
    ctx = wg.Context(plans.N, plans.q, plans.p, plans.dnum)
    for r in plans.rotations():
        key, parts, kl = plans.key(int(r))
        ctx.set_key(wg.WG_KEY_ROTATION, key, rotation=int(r), parts=parts, key_level=kl)
    return ctx


# (transform, stage, level): S2C runs at level 1 (stage 2 rescales), C2S at 12 (stage 1
# rescales to 11) and 11 (stage 3 rescales).
CASES = [(0, 0, 1), (0, 1, 1), (0, 2, 1), (1, 0, 12), (1, 1, 12), (1, 2, 11), (1, 3, 11)]


@pytest.mark.parametrize("which,stage,level", CASES)
def test_bsgs_stage_matches_reference(wg, plans, gpu_ctx, which, stage, level):
    import torch

    info = plans.stage(which, stage)
    N = plans.N
    assert info["qp_limbs"] == level + 1 + len(plans.p)
    st = wg.LtStage(gpu_ctx, level, info["indices"], info["diagonals"], info["baby"], info["slot_count"],
                    info["rescale"])
    rng = np.random.default_rng(100 * which + stage)
    count = 3
    qcol = np.repeat(plans.q[: level + 1], N)
    ins = [((rng.integers(0, 1 << 62, (level + 1) * N, dtype=np.uint64) % qcol).astype(np.uint64),
            (rng.integers(0, 1 << 62, (level + 1) * N, dtype=np.uint64) % qcol).astype(np.uint64))
           for _ in range(count)]
    db = [wg.to_device(b) for b, _ in ins]
    da = [wg.to_device(a) for _, a in ins]
    st.apply(db, da)
    torch.cuda.synchronize()
    for k, (b, a) in enumerate(ins):
        rb, ra, out_level = plans.apply_stage(which, stage, level, b, a)
        assert out_level == (level - 1 if info["rescale"] else level)
        n = (out_level + 1) * N
        gb, ga = wg.to_host(db[k])[:n], wg.to_host(da[k])[:n]
        assert (gb == rb).all(), (which, stage, k, int((gb != rb).sum()))
        assert (ga == ra).all(), (which, stage, k, int((ga != ra).sum()))
    st.close()


# Synthetic stage shapes at N = 2^12 against the oracle's restatement of the same evaluator:
# each shape isolates one part (baby 0 only, one baby rotation, one giant rotation, a mix).
SYN = [([0], 4, False), ([1], 4, False), ([4], 4, False), ([0, 1, 2, 5, 9, 12], 4, False),
       ([0, 1, 2, 5, 9, 12], 4, True), ([3, 2047, 2040], 8, False)]


@pytest.mark.parametrize("indices,baby,rescale", SYN)
def test_bsgs_synthetic_shapes_match_oracle(wg, oracle_mod, indices, baby, rescale):
    import torch

    O = oracle_mod
    N = 1 << 12
    p, q = O.find_primes([50, 50], [40, 45, 45, 45], N)
    o = O.OracleCtx(N, q, p, 2)
    ctx = wg.Context(N, q, p, 2)
    s = o.ternary(64, 9)
    slots = N // 2
    rots = sorted({i % baby for i in indices if i % baby} | {(i // baby) * baby for i in indices if i // baby})
    keys = {}
    for r in rots:
        keys[r] = o.rotation_key(s, r, 500 + r)
        ctx.set_key(wg.WG_KEY_ROTATION, keys[r], rotation=r)
    level = 3
    T = level + 1 + 2
    rng = np.random.default_rng(len(indices) + baby)
    mods = np.concatenate([q[: level + 1], p])
    diags = np.concatenate([(rng.integers(0, 1 << 62, T * N, dtype=np.uint64) % np.repeat(mods, N)).astype(np.uint64)
                            for _ in indices])
    st = wg.LtStage(ctx, level, indices, diags, baby, slots, rescale)
    ins = [(o.uniform(level + 1, 10 + k), o.uniform(level + 1, 20 + k)) for k in range(2)]
    db = [wg.to_device(b) for b, _ in ins]
    da = [wg.to_device(a) for _, a in ins]
    st.apply(db, da)
    torch.cuda.synchronize()
    for k, (b, a) in enumerate(ins):
        ob, oa = o.lt_stage(level, indices, diags, baby, slots, rescale, keys, b, a)
        n = ob.size
        gb, ga = wg.to_host(db[k])[:n], wg.to_host(da[k])[:n]
        assert (gb == ob).all() and (ga == oa).all(), (indices, baby, k, int((gb != ob).sum()), int((ga != oa).sum()))
