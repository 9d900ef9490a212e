"""Pin the C oracle (oracle/ckks_oracle.c) against the reference compiled from its own sources.

Both run on the same inputs; switching keys are the reference's own (exported from its
CKKSContext), so every residue must agree bit for bit.  Skipped where the reference sources
are not available (the GPU machines); the golden fixtures cover those.
"""
import numpy as np
import pytest

from params import CONFIG1, SMALL, WALSH15


def _ctxs(O, prm, rotations=(1,)):
    N = 1 << prm["logN"]
    R = O.RefCtx(N, prm["q_bits"], prm["p_bits"], prm["dnum"], h=prm["h"], rotations=list(rotations))
    o = O.OracleCtx(N, R.q, R.p, prm["dnum"])
    return N, R, o


def _uniform(rng, q, N, limbs):
    return np.concatenate([rng.integers(0, int(q[i]), N, dtype=np.uint64) for i in range(limbs)])


@pytest.mark.parametrize("prm", [CONFIG1, WALSH15] + SMALL)
def test_prime_chain(ref_mod, prm):
    O = ref_mod
    N = 1 << prm["logN"]
    p, q = O.find_primes(prm["p_bits"], prm["q_bits"], N)
    R = O.ref()
    pr = np.zeros(len(p), np.uint64)
    qr = np.zeros(len(q), np.uint64)
    assert R.ref_find_primes(np.array(prm["p_bits"], np.uint64), len(p), np.array(prm["q_bits"], np.uint64),
                             len(q), N, pr, qr) == 0
    assert (p == pr).all() and (q == qr).all()
    assert len(set(p.tolist() + q.tolist())) == len(p) + len(q)


@pytest.mark.parametrize("logN", [10, 12, 14, 15])
def test_ntt_tables(ref_mod, logN):
    import ctypes as C

    O = ref_mod
    N = 1 << logN
    p, q = O.find_primes([61], [36, 50], N)
    for m in list(q) + list(p):
        mine = O.ntt_tables(N, m)
        f, fs, i, is_ = (np.zeros(N, np.uint64) for _ in range(4))
        is_ = np.zeros(N + 1, np.uint64)
        ninv = C.c_uint64()
        bar = np.zeros(2, np.uint64)
        assert O.ref().ref_ntt_tables(N, int(m), f, fs, i, is_, C.byref(ninv), bar) == 0
        for a, b in zip(mine[:4], (f, fs, i, is_)):
            assert (a == b).all()
        assert mine[4] == ninv.value


@pytest.mark.parametrize("prm", SMALL)
def test_ops_small(ref_mod, prm):
    N, R, o = _ctxs(ref_mod, prm, rotations=(1, 3, -2))
    rng = np.random.default_rng(prm["logN"])
    L = len(R.q)
    x = _uniform(rng, R.q, N, L)
    assert (R.ntt(x) == o.ntt(x)).all()
    assert (R.ntt(x, inverse=True) == o.ntt(x, inverse=True)).all()
    rot_keys = {r: R.key(0, r) for r in (1, 3, -2)}
    conj_key, _, kl = R.key(1)
    relin_key, _, _ = R.key(2)
    for level in sorted({L - 1, L // 2, 1, 0}):
        b, a = _uniform(rng, R.q, N, level + 1), _uniform(rng, R.q, N, level + 1)
        for r, (k, _, kl) in rot_keys.items():
            rb, ra = R.rotate(level, b, a, r)
            ob, oa = o.rotate(level, b, a, k, r, key_level=kl)
            assert (rb == ob).all() and (ra == oa).all(), ("rotate", level, r)
        rb, ra = R.conjugate(level, b, a)
        ob, oa = o.conjugate(level, b, a, conj_key, key_level=kl)
        assert (rb == ob).all() and (ra == oa).all(), ("conjugate", level)
        # raw key switch in both combine modes
        kt = _uniform(rng, R.q, N, level + 1)
        k, parts, kl = rot_keys[1]
        for b_add, a_add in ((0, 0), (1, 1)):
            rb, ra = R.keyswitch(level, kt, k, parts, kl, b, a, b_add, a_add)
            ob, oa = o.keyswitch(level, kt, k, b, a, b_add, a_add, key_level=kl)
            assert (rb == ob).all() and (ra == oa).all(), ("keyswitch", level, b_add)
        b2, a2 = _uniform(rng, R.q, N, level + 1), _uniform(rng, R.q, N, level + 1)
        rm = R.mul(level, b, a, b2, a2)
        om = o.mul(level, b, a, b2, a2)
        assert all((u == v).all() for u, v in zip(rm, om)), ("mul", level)
        rr = R.relin(level, *rm)
        orr = o.relin(level, *om, relin_key, key_level=kl)
        assert (rr[0] == orr[0]).all() and (rr[1] == orr[1]).all(), ("relin", level)
        if level > 0:
            rs = R.rescale(level, list(rr))
            os_ = o.rescale(level, list(orr))
            assert all((u == v).all() for u, v in zip(rs, os_)), ("rescale", level)
        hr = R.hoisted_rotations(level, b, a, [1, 3, -2])
        for j, r in enumerate((1, 3, -2)):
            ob, oa = o.rotate(level, b, a, rot_keys[r][0], r, key_level=kl)
            assert (hr[j, 0] == ob).all() and (hr[j, 1] == oa).all(), ("hoisted", level, r)


def test_config1_rotation(ref_mod):
    """Config 1 at full size: N = 2^14, 16 Q limbs, dnum = 4, rotation by +1."""
    N, R, o = _ctxs(ref_mod, CONFIG1, rotations=(1,))
    rng = np.random.default_rng(1)
    L = len(R.q)
    x = _uniform(rng, R.q, N, L)
    assert (R.ntt(x) == o.ntt(x)).all()
    assert (R.ntt(x, inverse=True) == o.ntt(x, inverse=True)).all()
    k, _, kl = R.key(0, 1)
    b, a = _uniform(rng, R.q, N, L), _uniform(rng, R.q, N, L)
    rb, ra = R.rotate(L - 1, b, a, 1)
    ob, oa = o.rotate(L - 1, b, a, k, 1, key_level=kl)
    assert (rb == ob).all() and (ra == oa).all()


def test_walsh15_chain_ops(ref_mod):
    """The walsh15 modulus chain at N = 2^15: mul, relin, rescale, rotate at several levels."""
    N, R, o = _ctxs(ref_mod, WALSH15, rotations=(512, -7))
    rng = np.random.default_rng(15)
    relin_key, _, kl = R.key(2)
    rk = {r: R.key(0, r)[0] for r in (512, -7)}
    for level, r in ((12, 512), (6, -7), (1, 512)):
        b, a = _uniform(rng, R.q, N, level + 1), _uniform(rng, R.q, N, level + 1)
        b2, a2 = _uniform(rng, R.q, N, level + 1), _uniform(rng, R.q, N, level + 1)
        rm = R.mul(level, b, a, b2, a2)
        om = o.mul(level, b, a, b2, a2)
        assert all((u == v).all() for u, v in zip(rm, om))
        rr = R.relin(level, *rm)
        orr = o.relin(level, *om, relin_key, key_level=kl)
        assert (rr[0] == orr[0]).all() and (rr[1] == orr[1]).all()
        rs = R.rescale(level, list(rr))
        os_ = o.rescale(level, list(orr))
        assert all((u == v).all() for u, v in zip(rs, os_))
        rb, ra = R.rotate(level - 1, rs[0], rs[1], r)
        ob, oa = o.rotate(level - 1, os_[0], os_[1], rk[r], r, key_level=kl)
        assert (rb == ob).all() and (ra == oa).all()


def test_bsgs_stages_match_reference(ref_mod):
    """The oracle's QP BSGS stage against the reference's own walsh15 S2C / C2S plans."""
    P = ref_mod.RefPlans()
    o = ref_mod.OracleCtx(P.N, P.q, P.p, P.dnum)
    keys = {int(r): P.key(int(r))[0] for r in P.rotations()}
    rng = np.random.default_rng(3)
    for which, stage, level in ((0, 0, 1), (0, 2, 1), (1, 1, 12), (1, 3, 11)):
        info = P.stage(which, stage)
        b, a = _uniform(rng, P.q, P.N, level + 1), _uniform(rng, P.q, P.N, level + 1)
        rb, ra, _ = P.apply_stage(which, stage, level, b, a)
        ob, oa = o.lt_stage(level, info["indices"], info["diagonals"], info["baby"], info["slot_count"],
                            info["rescale"], keys, b, a)
        assert (rb == ob).all() and (ra == oa).all(), (which, stage)


def test_bootstrap_boundary_steps_match_reference(oracle_mod, ref_mod):
    """ModRaise, the q0/p0 dense-to-sparse switch and the sparse-to-dense switch of the oracle
    against the reference's walsh15 bootstrapping context (its own keys)."""
    R = ref_mod.RefPlans(bootstrap_keys=True)
    N = R.N
    o = oracle_mod.OracleCtx(N, R.q, R.p, R.dnum)
    rng = np.random.default_rng(1)
    b = (rng.integers(0, 1 << 62, N, dtype=np.uint64) % R.q[0]).astype(np.uint64)
    a = (rng.integers(0, 1 << 62, N, dtype=np.uint64) % R.q[0]).astype(np.uint64)
    for tl in (12, 1):
        rb, ra = R.modraise(tl, b, a)
        ob, oa = o.modraise(tl, b, a)
        assert (rb == ob).all() and (ra == oa).all(), tl
    k3, _, _ = R.key(0, kind=3)
    rb, ra = R.dense_to_sparse(b, a)
    ob, oa = o.q0p0_switch(k3, b, a)
    assert (rb == ob).all() and (ra == oa).all()
    k4, _, kl = R.key(0, kind=4)
    lv = 5
    qc = np.repeat(R.q[: lv + 1], N)
    bb = (rng.integers(0, 1 << 62, (lv + 1) * N, dtype=np.uint64) % qc).astype(np.uint64)
    aa = (rng.integers(0, 1 << 62, (lv + 1) * N, dtype=np.uint64) % qc).astype(np.uint64)
    rb, ra = R.sparse_to_dense(lv, bb, aa)
    ob, oa = o.keyswitch(lv, aa, k4, bb, aa, True, False, key_level=kl)
    assert (rb == ob).all() and (ra == oa).all()
