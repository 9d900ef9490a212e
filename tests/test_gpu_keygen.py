"""Rotation, conjugation and relinearisation switching keys generated on the device
(wg_keygen_switch_key) on the walsh15 chain (N = 2^15, 13 Q limbs, 4 P limbs, dnum 3) with the
reference context's own secret:

* with the mask and noise given, the device key equals, word for word, the key the reference's
  construction (generate_rotation_key_hybrid, rotation_key_generation.cpp:92-199, and
  generate_conjugation_key_hybrid, conjugation_key_generation.cpp:63-167, encrypt_rlk_hybrid,
  relinearization_key_generation.cpp:131-199, and the bootstrapping secret switches of
  secret_key_generation.cpp:227-364, the dense-to-sparse one as the compact q0/p0 key) makes
  from the same
  mask and noise on its own NTT, pointwise, folding and Montgomery helpers (the harness passes
  them in place of its random draws);
* with mask and noise drawn on the device, a rotation (and a relinearisation) through the
  installed key and the same operation through the reference's key (its own random draws)
  decrypt to the same values: their difference under the secret is key-switching noise, far
  below the modulus."""
import numpy as np
import pytest

from params import WALSH15

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(wg, ref_mod):
    R = ref_mod.RefCtx(1 << WALSH15["logN"], WALSH15["q_bits"], WALSH15["p_bits"], WALSH15["dnum"],
                       h=WALSH15["h"], rotations=[1, 3])
    ctx = wg.Context(R.N, R.q, R.p, R.dnum)
    s = R.secret_coeffs()
    assert s is not None and int((s != 0).sum()) == WALSH15["h"]
    return R, ctx, s


@pytest.mark.parametrize("kind,rotation", [("rotation", 1), ("rotation", -512), ("conjugation", 0),
                                           ("relinearisation", 0)])
def test_key_from_given_mask_and_noise_matches_reference(wg, setup, kind, rotation):
    R, ctx, s = setup
    N, L, K = R.N, len(R.q), len(R.p)
    parts = ctx.parts(L - 1)
    rng = np.random.default_rng(7 + abs(rotation))
    mods = np.concatenate([R.q, R.p]).astype(np.uint64)
    a = (rng.integers(0, 1 << 62, (parts, L + K, N), dtype=np.uint64) % mods[None, :, None]).astype(np.uint64)
    e = np.round(rng.normal(0.0, 3.2, (parts, N))).astype(np.int64)
    ref_kind = {"rotation": 0, "conjugation": 1, "relinearisation": 2}[kind]
    want = R.switch_key_from_parts(ref_kind, rotation, s, a, e)
    wkind = {"rotation": wg.WG_KEY_ROTATION, "conjugation": wg.WG_KEY_CONJ, "relinearisation": wg.WG_KEY_RELIN}[kind]
    got = ctx.keygen_switch_key(wkind, rotation, s, a=a, e=e, want_key=True)
    assert got.size == want.size
    assert (got == want).all(), int((got != want).sum())


def _centered_limb0_error(R, s_ntt0, x, y):
    """(x_b - y_b) + (x_a - y_a) s on limb 0, back in coefficient form, centred: its largest
    magnitude in bits."""
    N, q0 = R.N, int(R.q[0])
    db = (x[0][:N].astype(object) - y[0][:N].astype(object)) % q0
    da = (x[1][:N].astype(object) - y[1][:N].astype(object)) % q0
    d = np.array([(u + v * w) % q0 for u, v, w in zip(db.tolist(), da.tolist(), s_ntt0.tolist())], dtype=np.uint64)
    c = R.ntt(d, inverse=True)
    cen = [int(v) if v < q0 // 2 else int(v) - q0 for v in c.tolist()]
    return max(abs(v) for v in cen).bit_length()


def test_sampled_key_rotates_like_the_reference_key(wg, setup, ref_mod):
    import torch

    R, ctx, s = setup
    N, level = R.N, 6
    ctx.keygen_switch_key(wg.WG_KEY_ROTATION, 3, s, seed=2026)
    n = (level + 1) * N
    rng = np.random.default_rng(3)
    qc = np.repeat(R.q[: level + 1], N)
    b = (rng.integers(0, 1 << 62, n, dtype=np.uint64) % qc).astype(np.uint64)
    a = (rng.integers(0, 1 << 62, n, dtype=np.uint64) % qc).astype(np.uint64)
    db, da = wg.to_device(b), wg.to_device(a)
    ctx.rotate(level, db, da, 3)
    torch.cuda.synchronize()
    got = (wg.to_host(db), wg.to_host(da))
    want = R.rotate(level, b, a, 3)
    sk = np.zeros(len(R.q) * N, np.uint64)
    ref_mod.ref().ref_ctx_secret(R.h, sk)
    bits = _centered_limb0_error(R, sk[:N].astype(object), got, want)
    assert bits < 20, bits  # random residues would reach the size of q0 (36 bits)
    # and the keys themselves differ (independent draws)
    assert not (got[1] == want[1]).all()


def test_sampled_relin_key_relinearises_like_the_reference_key(wg, setup, ref_mod):
    import torch

    R, ctx, s = setup
    N, level = R.N, 5
    ctx.keygen_switch_key(wg.WG_KEY_RELIN, 0, s, seed=77)
    n = (level + 1) * N
    rng = np.random.default_rng(5)
    qc = np.repeat(R.q[: level + 1], N)
    draw = lambda: (rng.integers(0, 1 << 62, n, dtype=np.uint64) % qc).astype(np.uint64)
    c0, c1, c2 = draw(), draw(), draw()
    d0, d1, d2 = wg.to_device(c0), wg.to_device(c1), wg.to_device(c2)
    ctx.relin(level, d0, d1, d2)
    torch.cuda.synchronize()
    got = (wg.to_host(d0), wg.to_host(d1))
    want = R.relin(level, c0, c1, c2)
    sk = np.zeros(len(R.q) * N, np.uint64)
    ref_mod.ref().ref_ctx_secret(R.h, sk)
    bits = _centered_limb0_error(R, sk[:N].astype(object), got, want[:2])
    assert bits < 20, bits


@pytest.mark.parametrize("kind", ["sparse_to_dense", "dense_to_sparse"])
def test_secret_switch_key_matches_reference(wg, setup, kind):
    R, ctx, s = setup
    N, L, K = R.N, len(R.q), len(R.p)
    rng = np.random.default_rng(11 if kind == "sparse_to_dense" else 13)
    sparse = np.zeros(N, np.int8)
    sparse[rng.choice(N, 32, replace=False)] = rng.choice([-1, 1], 32).astype(np.int8)
    if kind == "sparse_to_dense":
        source, target, ref_kind, wkind = sparse, s, 4, wg.WG_KEY_SPARSE_TO_DENSE
        mods = np.concatenate([R.q, R.p]).astype(np.uint64)
        parts = ctx.parts(L - 1)
    else:
        source, target, ref_kind, wkind = s, sparse, 3, wg.WG_KEY_DENSE_TO_SPARSE
        mods = np.array([R.q[0], R.p[0]], dtype=np.uint64)
        parts = 1
    a = (rng.integers(0, 1 << 62, (parts, mods.size, N), dtype=np.uint64) % mods[None, :, None]).astype(np.uint64)
    e = np.round(rng.normal(0.0, 3.2, (parts, N))).astype(np.int64)
    want = R.switch_key_from_parts(ref_kind, 0, source, a, e, target=target)
    got = ctx.keygen_secret_switch(wkind, source, target, a=a, e=e, want_key=True)
    assert got.size == want.size
    assert (got == want).all(), int((got != want).sum())


def test_encrypt_from_given_mask_and_noise_matches_reference(wg, setup):
    import torch

    R, ctx, s = setup
    N, level, count = R.N, 4, 3
    n = (level + 1) * N
    rng = np.random.default_rng(17)
    qc = np.repeat(R.q[: level + 1], N)
    draw = lambda: (rng.integers(0, 1 << 62, n, dtype=np.uint64) % qc).astype(np.uint64)
    pts = [draw() for _ in range(count)]
    a = np.stack([draw() for _ in range(count)])
    e = np.round(rng.normal(0.0, 3.2, (count, N))).astype(np.int64)
    outs = [(torch.zeros(n, dtype=torch.int64, device="cuda"), torch.zeros(n, dtype=torch.int64, device="cuda"))
            for _ in range(count)]
    ctx.encrypt_symmetric(level, [wg.to_device(p) for p in pts], s, outs, a=a, e=e)
    torch.cuda.synchronize()
    for i in range(count):
        wb, wa = R.encrypt_from_parts(level, pts[i], s, a[i], e[i])
        assert (wg.to_host(outs[i][0]) == wb).all(), i
        assert (wg.to_host(outs[i][1]) == wa).all(), i
