"""The EvalMod bootstrap on the device against the reference's
ckks_batch_bootstrap_evalmod_from_complex_packed, both on the walsh15 bootstrapping context the
reference builds (its own S2C / C2S plans, rotation, conjugation, relinearisation and secret
switch keys, and the EvalMod series the context reports): SlotToCoeff, dense-to-sparse,
ModRaise, sparse-to-dense, CoeffToSlot, conjugate split and EvalMod, for a batch of packed
ciphertexts; both outputs must be identical residue for residue."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bts(ref_mod):
    return ref_mod.RefPlans(bootstrap_keys=True)


def test_bootstrap_evalmod_matches_reference(wg, bts):
    import torch

    info = bts.bts_info()
    N, K = bts.N, len(bts.p)
    ctx = wg.Context(N, bts.q, bts.p, bts.dnum)
    for kind, wkind in ((2, wg.WG_KEY_RELIN), (1, wg.WG_KEY_CONJ), (4, wg.WG_KEY_SPARSE_TO_DENSE)):
        key, parts, kl = bts.key(0, kind=kind)
        ctx.set_key(wkind, key, parts=parts, key_level=kl)
    ctx.set_key(wg.WG_KEY_DENSE_TO_SPARSE, bts.key(0, kind=3)[0])
    for r in bts.rotations():
        key, parts, kl = bts.key(int(r))
        ctx.set_key(wg.WG_KEY_ROTATION, key, rotation=int(r), parts=parts, key_level=kl)
    stages = []
    for which in (0, 1):
        lst = []
        for k in range(bts.stages(which)):
            st = bts.stage(which, k)
            level = st["qp_limbs"] - 1 - K
            lst.append(wg.LtStage(ctx, level, st["indices"], st["diagonals"], st["baby"], st["slot_count"],
                                  st["rescale"]))
        stages.append(lst)
    params = wg.BootstrapParams(info["s2c_depth"], info["depth"], info["evalmod_log_scale"], info["double_angle"],
                                info["active_slots"], info["slots"], info["scale"])
    level = info["s2c_depth"]
    full = (info["depth"] + 1) * N
    rng = np.random.default_rng(5)
    qc = np.repeat(bts.q[: level + 1], N)
    count = 2
    ins = [((rng.integers(0, 1 << 62, (level + 1) * N, dtype=np.uint64) % qc).astype(np.uint64),
            (rng.integers(0, 1 << 62, (level + 1) * N, dtype=np.uint64) % qc).astype(np.uint64)) for _ in range(count)]
    bs, as_ = [], []
    for b, a in ins:
        tb = torch.zeros(full, dtype=torch.int64, device="cuda")
        ta = torch.zeros(full, dtype=torch.int64, device="cuda")
        tb[: b.size] = wg.to_device(b)
        ta[: a.size] = wg.to_device(a)
        bs.append(tb)
        as_.append(ta)
    mk = lambda: torch.zeros(full, dtype=torch.int64, device="cuda")
    out0 = [(mk(), mk()) for _ in range(count)]
    out1 = [(mk(), mk()) for _ in range(count)]
    lvl, sc = ctx.bootstrap_evalmod(params, stages[0], stages[1], info["coeffs"], bs, as_, out0, out1)
    torch.cuda.synchronize()
    for i, (b, a) in enumerate(ins):
        (r0b, r0a), (r1b, r1a), rl, rs = bts.bootstrap_evalmod(level, info["scale"], b, a)
        assert (lvl, sc) == (rl, rs)
        n = (rl + 1) * N
        for got, want, name in ((out0[i][0], r0b, "out0.b"), (out0[i][1], r0a, "out0.a"), (out1[i][0], r1b, "out1.b"),
                                (out1[i][1], r1a, "out1.a")):
            g = wg.to_host(got)[:n]
            assert (g == want).all(), (i, name, int((g != want).sum()))
