"""Device library (libwalshgpu.so, through its C ABI) against the reference and the oracle.

Every comparison is bit for bit on raw uint64 residues:
  * golden fixtures produced by the reference itself (its own keys, tests/golden/);
  * the oracle on seeded inputs at small sizes, at config-1 size (N = 2^14, 16 limbs,
    dnum = 4) and on the walsh15 chain (N = 2^15, 13 limbs, dnum = 3).
"""
import numpy as np
import pytest

from params import CONFIG1, SMALL, WALSH15

pytestmark = pytest.mark.gpu


def _dev(wg, x):
    return wg.to_device(x)


def _host(wg, t):
    import torch

    torch.cuda.synchronize()
    return wg.to_host(t)


def _gctx(wg, g):
    N = int(g["N"][0])
    ctx = wg.Context(N, g["q"], g["p"], int(g["dnum"][0]))
    kl = int(g["key_level"][0])
    parts = int(g["key_parts"][0])
    ctx.set_key(wg.WG_KEY_ROTATION, g["rot_key"], rotation=int(g["rotation"][0]), parts=parts, key_level=kl)
    ctx.set_key(wg.WG_KEY_CONJ, g["conj_key"], parts=parts, key_level=kl)
    ctx.set_key(wg.WG_KEY_RELIN, g["relin_key"], parts=parts, key_level=kl)
    return ctx


def test_golden_ntt(wg, golden):
    g = golden
    ctx = _gctx(wg, g)
    L = len(g["q"])
    x = _dev(wg, g["ntt_in"])
    ctx.ntt_forward(x, L)
    assert (_host(wg, x) == g["ntt_fwd"]).all()
    y = _dev(wg, g["ntt_in"])
    ctx.ntt_inverse(y, L)
    assert (_host(wg, y) == g["ntt_inv"]).all()


def test_golden_ops(wg, golden):
    import torch

    g = golden
    ctx = _gctx(wg, g)
    N = int(g["N"][0])
    L = len(g["q"])
    rot = int(g["rotation"][0])
    for level in (L - 1, 2):
        n = (level + 1) * N
        b, a = _dev(wg, g[f"l{level}_b"]), _dev(wg, g[f"l{level}_a"])
        ctx.rotate(level, b, a, rot)
        assert (_host(wg, b) == g[f"l{level}_rot_b"]).all() and (_host(wg, a) == g[f"l{level}_rot_a"]).all()
        b, a = _dev(wg, g[f"l{level}_b"]), _dev(wg, g[f"l{level}_a"])
        ctx.conjugate(level, b, a)
        assert (_host(wg, b) == g[f"l{level}_conj_b"]).all() and (_host(wg, a) == g[f"l{level}_conj_a"]).all()
        b, a = _dev(wg, g[f"l{level}_b"]), _dev(wg, g[f"l{level}_a"])
        b2, a2 = _dev(wg, g[f"l{level}_b2"]), _dev(wg, g[f"l{level}_a2"])
        c2 = torch.empty(n, dtype=torch.int64, device="cuda")
        ctx.mul(level, b, a, b2, a2, c2)
        assert (_host(wg, b) == g[f"l{level}_mul_c0"]).all()
        assert (_host(wg, a) == g[f"l{level}_mul_c1"]).all()
        assert (_host(wg, c2) == g[f"l{level}_mul_c2"]).all()
        ctx.relin(level, b, a, c2)
        assert (_host(wg, b) == g[f"l{level}_relin_b"]).all() and (_host(wg, a) == g[f"l{level}_relin_a"]).all()
        ct = torch.stack([b, a])
        ctx.rescale(level, ct, npolys=2, stride=n)
        out = _host(wg, ct)
        assert (out[0, : level * N] == g[f"l{level}_rescale_b"]).all()
        assert (out[1, : level * N] == g[f"l{level}_rescale_a"]).all()


def _oracle_setup(O, wg, prm, rotations, seed=5):
    N = 1 << prm["logN"]
    p, q = O.find_primes(prm["p_bits"], prm["q_bits"], N)
    o = O.OracleCtx(N, q, p, prm["dnum"])
    ctx = wg.Context(N, q, p, prm["dnum"])
    s = o.ternary(min(prm["h"], N // 4), seed)
    keys = {}
    for r in rotations:
        keys[r] = o.rotation_key(s, r, 100 + r % 1000)
        ctx.set_key(wg.WG_KEY_ROTATION, keys[r], rotation=r)
    conj = o.conjugation_key(s, 7)
    relin = o.relin_key(s, 9)
    ctx.set_key(wg.WG_KEY_CONJ, conj)
    ctx.set_key(wg.WG_KEY_RELIN, relin)
    return N, o, ctx, keys, conj, relin


@pytest.mark.parametrize("fusion", [1, 2])
@pytest.mark.parametrize("prm", SMALL)
def test_small_sets_against_oracle(wg, oracle_mod, prm, fusion):
    """Every operation on one ciphertext at several levels against the oracle; fusion 1 (the
    default) runs single ciphertexts through the separate launches, 2 forces the fused
    key-switch and rescale kernels."""
    import torch

    O = oracle_mod
    rots = (1, 3, -2)
    N, o, ctx, keys, conj, relin = _oracle_setup(O, wg, prm, rots)
    ctx.set_ntt_fusion(fusion)
    L = o.nq
    x = o.uniform(L, 11)
    d = _dev(wg, x)
    ctx.ntt_forward(d, L)
    assert (_host(wg, d) == o.ntt(x)).all()
    ctx.ntt_inverse(d, L)
    assert (_host(wg, d) == x).all()
    # P-basis limbs
    pp = np.concatenate([np.random.default_rng(1).integers(0, int(m), N, dtype=np.uint64) for m in o.p])
    dp = _dev(wg, pp)
    ctx.ntt_forward(dp, len(o.p), basis=1)
    assert (_host(wg, dp) == o.ntt(pp, which=1)).all()
    for level in sorted({L - 1, L // 2, 1, 0}):
        n = (level + 1) * N
        b, a = o.uniform(level + 1, 20 + level), o.uniform(level + 1, 40 + level)
        for r in rots:
            db, da = _dev(wg, b), _dev(wg, a)
            ctx.rotate(level, db, da, r)
            ob, oa = o.rotate(level, b, a, keys[r], r)
            assert (_host(wg, db) == ob).all() and (_host(wg, da) == oa).all(), ("rotate", level, r)
        db, da = _dev(wg, b), _dev(wg, a)
        ctx.conjugate(level, db, da)
        ob, oa = o.conjugate(level, b, a, conj)
        assert (_host(wg, db) == ob).all() and (_host(wg, da) == oa).all(), ("conjugate", level)
        kt = o.uniform(level + 1, 77)
        for b_add, a_add in ((0, 0), (1, 1), (1, 0)):
            db, da = _dev(wg, b), _dev(wg, a)
            ctx.keyswitch(level, _dev(wg, kt), wg.WG_KEY_ROTATION, db, da, b_add, a_add, rotation=3)
            ob, oa = o.keyswitch(level, kt, keys[3], b, a, b_add, a_add)
            assert (_host(wg, db) == ob).all() and (_host(wg, da) == oa).all(), ("keyswitch", level)
        b2, a2 = o.uniform(level + 1, 60), o.uniform(level + 1, 61)
        db, da, db2, da2 = _dev(wg, b), _dev(wg, a), _dev(wg, b2), _dev(wg, a2)
        c2 = torch.empty(n, dtype=torch.int64, device="cuda")
        ctx.mul(level, db, da, db2, da2, c2)
        oc0, oc1, oc2 = o.mul(level, b, a, b2, a2)
        assert (_host(wg, db) == oc0).all() and (_host(wg, da) == oc1).all() and (_host(wg, c2) == oc2).all()
        ctx.relin(level, db, da, c2)
        or0, or1 = o.relin(level, oc0, oc1, oc2, relin)
        assert (_host(wg, db) == or0).all() and (_host(wg, da) == or1).all(), ("relin", level)
        if level > 0:
            ctx.rescale(level, db)
            ctx.rescale(level, da)
            os0, os1 = o.rescale(level, [or0, or1])
            assert (_host(wg, db)[: level * N] == os0).all() and (_host(wg, da)[: level * N] == os1).all()
        # add / sub
        dx, dy = _dev(wg, b), _dev(wg, b2)
        ctx.add(level, dx, dy)
        qq = np.repeat(o.q[: level + 1], N)
        assert (_host(wg, dx) == (b + b2) % qq).all()
        ctx.sub(level, dx, dy)
        assert (_host(wg, dx) == b).all()
        # several rotations of one ciphertext
        out = torch.empty(len(rots) * 2 * n, dtype=torch.int64, device="cuda")
        ctx.rotate_many(level, _dev(wg, b), _dev(wg, a), list(rots), out)
        ho = _host(wg, out).reshape(len(rots), 2, n)
        for j, r in enumerate(rots):
            ob, oa = o.rotate(level, b, a, keys[r], r)
            assert (ho[j, 0] == ob).all() and (ho[j, 1] == oa).all()


def test_config1_ntt_and_rotation(wg, oracle_mod):
    """Config 1: N = 2^14, 16 Q limbs; forward+inverse NTT of all limbs, rotation by +1."""
    N, o, ctx, keys, _, _ = _oracle_setup(oracle_mod, wg, CONFIG1, (1,))
    L = o.nq
    x = o.uniform(L, 123)
    d = _dev(wg, x)
    ctx.ntt_forward(d, L)
    fwd = _host(wg, d)
    assert (fwd == o.ntt(x)).all()
    ctx.ntt_inverse(d, L)
    assert (_host(wg, d) == x).all()
    b, a = o.uniform(L, 5), o.uniform(L, 6)
    db, da = _dev(wg, b), _dev(wg, a)
    ctx.rotate(L - 1, db, da, 1)
    ob, oa = o.rotate(L - 1, b, a, keys[1], 1)
    assert (_host(wg, db) == ob).all() and (_host(wg, da) == oa).all()


def test_trim_gives_back_scratch(wg, oracle_mod):
    """wg_ctx_trim frees the stream's scratch (device free memory rises by at least four
    ciphertext polynomials' worth: the key switch's digits alone are larger) and the context
    keeps working: a rotation before and after, bit-exact."""
    import torch

    N, o, ctx, keys, _, _ = _oracle_setup(oracle_mod, wg, CONFIG1, (1,))
    L = o.nq
    b, a = o.uniform(L, 5), o.uniform(L, 6)
    ob, oa = o.rotate(L - 1, b, a, keys[1], 1)
    for _ in range(2):
        db, da = _dev(wg, b), _dev(wg, a)
        ctx.rotate(L - 1, db, da, 1)
        assert (_host(wg, db) == ob).all() and (_host(wg, da) == oa).all()
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        ctx.trim()
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] - free0 >= 4 * 8 * L * N


@pytest.mark.parametrize("count,nrot", [(16, 4), (64, 16)])
def test_walsh15_batched_ops(wg, oracle_mod, count, nrot):
    """Config 2: walsh15 chain, ciphertexts at seeded levels 1..12, each mul + relin + rescale +
    rotate by a seeded index, through the batched entry point, bit-exact; at the benchmark's 64
    ciphertexts and a smaller batch."""
    import torch

    rng = np.random.default_rng(2 + count)
    # distinct rotations modulo the N/2 slots (-512 k and 512 (32 - k) would share one Galois
    # element, hence one key slot on the device, while the oracle is handed two different keys)
    pool = [512 * k for k in range(1, 16)] + [-512 * k for k in range(1, 16)]
    rots = [int(r) for r in rng.choice(pool, nrot, replace=False)]
    N, o, ctx, keys, _, relin = _oracle_setup(oracle_mod, wg, WALSH15, rots)
    levels = rng.integers(1, 13, count)
    ct_rots = [rots[i % len(rots)] for i in range(count)]
    L = o.nq
    stride = L * N
    xb = np.concatenate([o.uniform(L, 1000 + i) for i in range(count)])
    xa = np.concatenate([o.uniform(L, 2000 + i) for i in range(count)])
    yb = np.concatenate([o.uniform(L, 3000 + i) for i in range(count)])
    ya = np.concatenate([o.uniform(L, 4000 + i) for i in range(count)])
    dxb, dxa, dyb, dya = (_dev(wg, v) for v in (xb, xa, yb, ya))
    sl = lambda t, i: t[i * stride:(i + 1) * stride]
    n0 = wg.launch_count()
    ctx.batch_mul_relin_rescale_rotate(levels, [sl(dxb, i) for i in range(count)], [sl(dxa, i) for i in range(count)],
                                       [sl(dyb, i) for i in range(count)], [sl(dya, i) for i in range(count)], ct_rots)
    batch_launches = wg.launch_count() - n0
    gb, ga = _host(wg, dxb), _host(wg, dxa)
    # the live limbs of every result (levels[i] limbs after the rescale): the dropped limb is
    # scratch that each path leaves in its own intermediate form
    live = np.zeros(count * stride, dtype=bool)
    for i in range(count):
        live[i * stride:i * stride + int(levels[i]) * N] = True
    same = lambda x, y: (_host(wg, x)[live] == y[live]).all()
    # the plain per-operation path gives the same residues
    pxb, pxa = _dev(wg, xb), _dev(wg, xa)
    ctx.batch_mul_relin_rescale_rotate(levels, [sl(pxb, i) for i in range(count)], [sl(pxa, i) for i in range(count)],
                                       [sl(dyb, i) for i in range(count)], [sl(dya, i) for i in range(count)], ct_rots,
                                       plain=True)
    assert same(pxb, gb) and same(pxa, ga)
    # the base changes and final steps as separate launches instead of inside the NTT phases
    ctx.set_ntt_fusion(False)
    uxb, uxa = _dev(wg, xb), _dev(wg, xa)
    ctx.batch_mul_relin_rescale_rotate(levels, [sl(uxb, i) for i in range(count)], [sl(uxa, i) for i in range(count)],
                                       [sl(dyb, i) for i in range(count)], [sl(dya, i) for i in range(count)], ct_rots)
    ctx.set_ntt_fusion(True)
    assert same(uxb, gb) and same(uxa, ga)
    # the graph-captured plan over its own buffers: same residues, replayable
    gxb, gxa = _dev(wg, xb), _dev(wg, xa)
    plan = wg.BatchPlan(ctx, levels, [sl(gxb, i) for i in range(count)], [sl(gxa, i) for i in range(count)],
                        [sl(dyb, i) for i in range(count)], [sl(dya, i) for i in range(count)], ct_rots)
    n0 = wg.launch_count()
    for _ in range(2):
        gxb.copy_(_dev(wg, xb))
        gxa.copy_(_dev(wg, xa))
        plan.launch()
        assert same(gxb, gb) and same(gxa, ga)
    # a replay runs (and counts) the kernels of one batched call: one launch per stage
    assert wg.launch_count() - n0 == 2 * batch_launches and batch_launches < 40
    plan.close()
    ob, oa = xb.copy(), xa.copy()
    o.batched_ops(levels, ob, oa, yb, ya, relin, [keys[r] for r in ct_rots], ct_rots, stride, 8)
    for i in range(count):
        n = int(levels[i]) * N
        assert (gb[i * stride:i * stride + n] == ob[i * stride:i * stride + n]).all(), i
        assert (ga[i * stride:i * stride + n] == oa[i * stride:i * stride + n]).all(), i


def test_errors_follow_reference_conventions(wg, oracle_mod):
    import torch

    N, o, ctx, keys, _, _ = _oracle_setup(oracle_mod, wg, SMALL[0], (1,))
    b = torch.zeros(o.nq * N, dtype=torch.int64, device="cuda")
    a = torch.zeros_like(b)
    with pytest.raises(wg.InvalidArgument):
        ctx.rotate(o.nq, b, a, 1)  # level beyond the chain
    with pytest.raises(wg.WalshGpuError) as e:
        ctx.rotate(0, b, a, 5)  # no key for this rotation
    assert e.value.code == -2
    with pytest.raises(wg.InvalidArgument):
        ctx.rescale(0, b)
    ctx.rotate(0, b, a, N // 2)  # rotation by a multiple of the slot count is a no-op
