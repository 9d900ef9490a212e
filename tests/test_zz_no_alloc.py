"""wg_rotate_noalloc: the rotation for callers that cannot allocate device memory when they
rotate (memory already claimed by another allocator, loops that must avoid allocation-induced
synchronisation).  Its key-switch scratch is the library's fixed 32 MiB static device array
instead of per-stream workspace.

Checked through the C ABI, bit for bit, against wg_rotate and against the oracle on two calls in
a row (the array keeps the previous call's contents between them); at the level whose scratch
need is exactly the array's 4 Mi words (accepted) and the level above (rejected, buffers left
as they were); and with the device's free memory and the caching allocator's counters unchanged
across calls.  This file is collected last so a failure here never hides the other tests; it
also passes on its own.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SCRATCH_WORDS = 4 << 20  # the static array's size in 64-bit words


def _setup(wg, O, logN, q_bits, p_bits, dnum, rotations):
    N = 1 << logN
    p, q = O.find_primes(p_bits, q_bits, N)
    o = O.OracleCtx(N, q, p, dnum)
    ctx = wg.Context(N, q, p, dnum)
    s = o.ternary(64, 3)
    keys = {}
    for r in rotations:
        keys[r] = o.rotation_key(s, r, 40 + r)
        ctx.set_key(wg.WG_KEY_ROTATION, keys[r], rotation=r)
    return N, o, ctx, keys


def _workspace_words(N, level, K, dnum, nq):
    """Key-switch scratch of one rotation: N x (L + B (L + K) + 2 (L + K) + 2 L) words."""
    alpha = (nq + dnum - 1) // dnum
    L = level + 1
    B = min(dnum, (L + alpha - 1) // alpha)
    T = L + K
    return N * (L + B * T + 2 * T + 2 * L)


def _memory_counters(torch):
    torch.cuda.synchronize()
    free, _ = torch.cuda.mem_get_info()
    return free, torch.cuda.memory_allocated(), torch.cuda.memory_reserved()


def test_rotate_noalloc_matches_rotate_and_oracle(wg, oracle_mod):
    import torch

    N, o, ctx, keys = _setup(wg, oracle_mod, 15, [36, 61, 42, 42] + [38] * 7 + [50, 50], [61] * 4, 3,
                             (512, -3))
    L = o.nq
    for call, (level, rot) in enumerate(((L - 1, 512), (5, -3))):
        b, a = o.uniform(level + 1, 300 + call), o.uniform(level + 1, 400 + call)
        rb, ra = wg.to_device(b), wg.to_device(a)
        ctx.rotate(level, rb, ra, rot)
        nb, na = wg.to_device(b), wg.to_device(a)
        ctx.rotate_noalloc(level, nb, na, rot)
        torch.cuda.synchronize()
        ob, oa = o.rotate(level, b, a, keys[rot], rot)
        assert (wg.to_host(nb) == wg.to_host(rb)).all(), call
        assert (wg.to_host(na) == wg.to_host(ra)).all(), call
        assert (wg.to_host(nb) == ob).all(), call
        assert (wg.to_host(na) == oa).all(), call


def test_rotate_noalloc_allocates_no_device_memory(wg, oracle_mod):
    import torch

    N, o, ctx, keys = _setup(wg, oracle_mod, 14, [50] * 8, [55] * 2, 4, (7,))
    level = 7
    b, a = o.uniform(level + 1, 11), o.uniform(level + 1, 12)
    nb, na = wg.to_device(b), wg.to_device(a)
    ctx.rotate_noalloc(level, nb, na, 7)  # first call on the device: address lookup, kernels loaded
    before = _memory_counters(torch)
    for _ in range(3):
        ctx.rotate_noalloc(level, nb, na, 7)
    after = _memory_counters(torch)
    assert after == before, (before, after)
    # four rotations by 7 in a row equal the oracle's
    ob, oa = b, a
    for _ in range(4):
        ob, oa = o.rotate(level, ob, oa, keys[7], 7)
    assert (wg.to_host(nb) == ob).all() and (wg.to_host(na) == oa).all()


def test_rotate_noalloc_limit_is_exact(wg, oracle_mod):
    import torch

    # N = 2^15, 11 Q limbs, 4 P limbs, dnum 6 (digits of 2 limbs): level 9 needs exactly
    # 4 Mi words of scratch, level 10 needs 800 Ki words more.
    logN, q_bits, p_bits, dnum = 15, [50] * 11, [55] * 4, 6
    N, o, ctx, keys = _setup(wg, oracle_mod, logN, q_bits, p_bits, dnum, (1,))
    K, nq = len(p_bits), len(q_bits)
    assert _workspace_words(N, 9, K, dnum, nq) == SCRATCH_WORDS
    assert _workspace_words(N, 10, K, dnum, nq) > SCRATCH_WORDS

    level = 9
    b, a = o.uniform(level + 1, 21), o.uniform(level + 1, 22)
    nb, na = wg.to_device(b), wg.to_device(a)
    ctx.rotate_noalloc(level, nb, na, 1)
    torch.cuda.synchronize()
    ob, oa = o.rotate(level, b, a, keys[1], 1)
    assert (wg.to_host(nb) == ob).all() and (wg.to_host(na) == oa).all()

    level = 10
    b, a = o.uniform(level + 1, 23), o.uniform(level + 1, 24)
    nb, na = wg.to_device(b), wg.to_device(a)
    with pytest.raises(wg.InvalidArgument):
        ctx.rotate_noalloc(level, nb, na, 1)
    torch.cuda.synchronize()
    assert (wg.to_host(nb) == b).all() and (wg.to_host(na) == a).all()


def test_rotate_noalloc_rejects_levels_beyond_the_static_scratch(wg, oracle_mod):
    import torch

    # N = 2^16 with 10 Q limbs and 4 P limbs needs ~50 MiB of key-switch scratch at the top level
    N, o, ctx, _ = _setup(wg, oracle_mod, 16, [50] * 10, [55] * 4, 3, (1,))
    b = torch.zeros(10 * N, dtype=torch.int64, device="cuda")
    a = torch.zeros_like(b)
    with pytest.raises(wg.InvalidArgument):
        ctx.rotate_noalloc(9, b, a, 1)
    ctx.rotate_noalloc(1, b[: 2 * N], a[: 2 * N], 1)  # a low level fits
    torch.cuda.synchronize()
