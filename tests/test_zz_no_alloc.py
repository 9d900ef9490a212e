"""wg_rotate_noalloc: the rotation for callers that cannot allocate device memory when they
rotate (memory already claimed by another allocator, loops that must avoid allocation-induced
synchronisation).  Its key-switch scratch is the
library's fixed 32 MiB static device array instead of per-stream workspace.

Checked through the C ABI against wg_rotate, bit for bit, on two calls in a row (the array
keeps the previous call's contents between them), plus the size-limit error.  This file is
collected last so a failure here never hides the other tests; it also passes on its own.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(wg, O, logN, q_bits, p_bits, dnum, rotations):
    N = 1 << logN
    p, q = O.find_primes(p_bits, q_bits, N)
    o = O.OracleCtx(N, q, p, dnum)
    ctx = wg.Context(N, q, p, dnum)
    s = o.ternary(64, 3)
    for r in rotations:
        ctx.set_key(wg.WG_KEY_ROTATION, o.rotation_key(s, r, 40 + r), rotation=r)
    return N, o, ctx


def test_rotate_noalloc_matches_rotate(wg, oracle_mod):
    import torch

    N, o, ctx, = _setup(wg, oracle_mod, 15, [36, 61, 42, 42] + [38] * 7 + [50, 50], [61] * 4, 3, (512, -3))
    L = o.nq
    for call, (level, rot) in enumerate(((L - 1, 512), (5, -3))):
        b, a = o.uniform(level + 1, 300 + call), o.uniform(level + 1, 400 + call)
        rb, ra = wg.to_device(b), wg.to_device(a)
        ctx.rotate(level, rb, ra, rot)
        nb, na = wg.to_device(b), wg.to_device(a)
        ctx.rotate_noalloc(level, nb, na, rot)
        torch.cuda.synchronize()
        assert (wg.to_host(nb) == wg.to_host(rb)).all(), call
        assert (wg.to_host(na) == wg.to_host(ra)).all(), call


def test_rotate_noalloc_rejects_levels_beyond_the_static_scratch(wg, oracle_mod):
    import torch

    # N = 2^16 with 10 Q limbs and 4 P limbs needs ~50 MiB of key-switch scratch at the top level
    N, o, ctx = _setup(wg, oracle_mod, 16, [50] * 10, [55] * 4, 3, (1,))
    b = torch.zeros(10 * N, dtype=torch.int64, device="cuda")
    a = torch.zeros_like(b)
    with pytest.raises(wg.InvalidArgument):
        ctx.rotate_noalloc(9, b, a, 1)
    ctx.rotate_noalloc(1, b[: 2 * N], a[: 2 * N], 1)  # a low level fits
    torch.cuda.synchronize()
