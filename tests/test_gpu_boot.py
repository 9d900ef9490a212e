"""Bootstrapping boundary steps on the device against the reference itself: ModRaise, the
level-0 dense-to-sparse switch through q0/p0 and the sparse-to-dense hybrid switch, with the
keys of the reference's walsh15 bootstrapping context (compiled from its own sources)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bts(ref_mod):
    return ref_mod.RefPlans(bootstrap_keys=True)


@pytest.fixture(scope="module")
def gpu_ctx(wg, bts):
    ctx = wg.Context(bts.N, bts.q, bts.p, bts.dnum)
    k3, _, _ = bts.key(0, kind=3)
    ctx.set_key(wg.WG_KEY_DENSE_TO_SPARSE, k3)
    k4, parts, kl = bts.key(0, kind=4)
    ctx.set_key(wg.WG_KEY_SPARSE_TO_DENSE, k4, parts=parts, key_level=kl)
    return ctx


def _uniform(rng, q, limbs, N):
    col = np.repeat(np.asarray(q[:limbs], dtype=np.uint64), N)
    return (rng.integers(0, 1 << 62, limbs * N, dtype=np.uint64) % col).astype(np.uint64)


@pytest.mark.parametrize("target", [12, 7, 1])
def test_modraise_matches_reference(wg, bts, gpu_ctx, target):
    import torch

    N = bts.N
    rng = np.random.default_rng(target)
    ins = [(_uniform(rng, bts.q, 1, N), _uniform(rng, bts.q, 1, N)) for _ in range(3)]
    n = (target + 1) * N
    db, da = [], []
    for b, a in ins:
        tb = torch.zeros(n, dtype=torch.int64, device="cuda")
        ta = torch.zeros(n, dtype=torch.int64, device="cuda")
        tb[:N] = wg.to_device(b)
        ta[:N] = wg.to_device(a)
        db.append(tb)
        da.append(ta)
    gpu_ctx.modraise(target, db, da)
    torch.cuda.synchronize()
    for k, (b, a) in enumerate(ins):
        rb, ra = bts.modraise(target, b, a)
        assert (wg.to_host(db[k]) == rb).all() and (wg.to_host(da[k]) == ra).all(), (target, k)


def test_dense_to_sparse_matches_reference(wg, bts, gpu_ctx):
    import torch

    N = bts.N
    rng = np.random.default_rng(7)
    ins = [(_uniform(rng, bts.q, 1, N), _uniform(rng, bts.q, 1, N)) for _ in range(4)]
    db = [wg.to_device(b) for b, _ in ins]
    da = [wg.to_device(a) for _, a in ins]
    gpu_ctx.dense_to_sparse(db, da)
    torch.cuda.synchronize()
    for k, (b, a) in enumerate(ins):
        rb, ra = bts.dense_to_sparse(b, a)
        assert (wg.to_host(db[k]) == rb).all() and (wg.to_host(da[k]) == ra).all(), k


def test_sparse_to_dense_matches_reference(wg, bts, gpu_ctx):
    import torch

    N = bts.N
    rng = np.random.default_rng(11)
    levels = [12, 3, 0, 9]
    ins = [(_uniform(rng, bts.q, lv + 1, N), _uniform(rng, bts.q, lv + 1, N)) for lv in levels]
    db = [wg.to_device(b) for b, _ in ins]
    da = [wg.to_device(a) for _, a in ins]
    gpu_ctx.sparse_to_dense(levels, db, da)
    torch.cuda.synchronize()
    for k, ((b, a), lv) in enumerate(zip(ins, levels)):
        rb, ra = bts.sparse_to_dense(lv, b, a)
        assert (wg.to_host(db[k]) == rb).all() and (wg.to_host(da[k]) == ra).all(), (k, lv)


def test_boundary_errors(wg, gpu_ctx, bts):
    import torch

    t = torch.zeros(bts.N, dtype=torch.int64, device="cuda")
    with pytest.raises(wg.InvalidArgument):
        gpu_ctx.modraise(0, [t], [t.clone()])
    with pytest.raises(wg.InvalidArgument):
        gpu_ctx.modraise(len(bts.q), [t], [t.clone()])
    bare = wg.Context(bts.N, bts.q, bts.p, bts.dnum)
    with pytest.raises(wg.WalshGpuError) as e:
        bare.dense_to_sparse([t], [t.clone()])
    assert e.value.code == -2
