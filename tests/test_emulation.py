"""CPU emulation of the device kernels against the oracle.

tests/emu/wg_emulate.cpp compiles the product's kernel bodies (wg_ntt.cuh, wg_keyswitch.cuh, wg_walsh.cuh)
and table builder with the host compiler and runs them thread by thread.  This checks index
logic, butterflies, HPS base changes and tables without a GPU; the GPU tests then check the
compiled kernels themselves.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from params import SMALL, WALSH15

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "aes-walsh-ckks_b200", "csrc")
u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")


@pytest.fixture(scope="module")
def emu(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("emu") / "libwgemu.so")
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-I", CSRC,
                    "-I", "/usr/local/cuda/include", os.path.join(ROOT, "tests", "emu", "wg_emulate.cpp"),
                    os.path.join(CSRC, "wg_tables.cpp"), os.path.join(CSRC, "wg_host.cpp"), "-o", out], check=True)
    E = C.CDLL(out)
    E.emu_create.restype = C.c_void_p
    E.emu_create.argtypes = [C.c_uint64, u64p, C.c_size_t, u64p, C.c_size_t, C.c_size_t]
    E.emu_destroy.argtypes = [C.c_void_p]
    E.emu_ntt.argtypes = [C.c_void_p, u64p, C.c_size_t, C.c_size_t, C.c_int, C.c_int]
    E.emu_set_ntt_geometry.argtypes = [C.c_int]
    E.emu_set_keyswitch_fusion.argtypes = [C.c_int]
    E.emu_rescale.argtypes = [C.c_void_p, C.c_size_t, u64p]
    E.emu_keyswitch.argtypes = [C.c_void_p, C.c_size_t, u64p, u64p, C.c_size_t, u64p, u64p, C.c_int, C.c_int,
                                C.c_uint64]
    return E


# one digit per Q limb: the key inner products and ModUp run over 8 parts of one limb each
MANY_DIGITS = dict(logN=10, q_bits=[40, 45, 45, 45, 50, 50, 50, 50], p_bits=[55], dnum=8, h=64)


@pytest.mark.parametrize("fused", [0, 1])
@pytest.mark.parametrize("prm", SMALL + [MANY_DIGITS])
def test_emulated_kernels_match_oracle(oracle_mod, emu, prm, fused):
    """NTT, key switch (rotation, relinearisation) and rescale at three levels; fused = 1 runs
    them as the device does by default: ModUp, ModDown and the rescale remainders inside the NTT
    column phases (wg_ksfuse.cuh), the combine and the rescale finish as the epilogue of the last
    row phase."""
    O = oracle_mod
    N = 1 << prm["logN"]
    p, q = O.find_primes(prm["p_bits"], prm["q_bits"], N)
    o = O.OracleCtx(N, q, p, prm["dnum"])
    h = emu.emu_create(N, q, len(q), p, len(p), prm["dnum"])
    emu.emu_set_keyswitch_fusion(fused)
    try:
        L = len(q)
        x = o.uniform(L, 5)
        y = x.copy()
        emu.emu_ntt(h, y, L, 0, 0, 0)
        assert (y == o.ntt(x)).all()
        z = y.copy()
        emu.emu_ntt(h, z, L, 0, 0, 1)
        assert (z == x).all()
        pp = np.concatenate([np.random.default_rng(3).integers(0, int(m), N, dtype=np.uint64) for m in p])
        pe = pp.copy()
        emu.emu_ntt(h, pe, len(p), 0, 1, 0)
        assert (pe == o.ntt(pp, which=1)).all()
        s = o.ternary(min(64, N // 4), 3)
        rk = o.rotation_key(s, 3, 11)
        rl = o.relin_key(s, 13)
        for level in sorted({L - 1, L // 2, 0}):
            n = (level + 1) * N
            b, a = x[:n].copy(), o.uniform(level + 1, 9)
            ob, oa = o.rotate(level, b, a, rk, 3)
            eb, ea = b.copy(), a.copy()
            emu.emu_keyswitch(h, level, a.copy(), rk, L - 1, eb, ea, 1, 0, o.galois(3))
            assert (eb == ob).all() and (ea == oa).all()
            c2 = o.uniform(level + 1, 21)
            r0, r1 = o.relin(level, b, a, c2, rl)
            e0, e1 = b.copy(), a.copy()
            emu.emu_keyswitch(h, level, c2, rl, L - 1, e0, e1, 1, 1, 0)
            assert (e0 == r0).all() and (e1 == r1).all()
            if level > 0:
                (os0,) = o.rescale(level, [r0])
                xs = r0.copy()
                emu.emu_rescale(h, level, xs)
                assert (xs[: level * N] == os0).all()
    finally:
        emu.emu_set_keyswitch_fusion(0)
        emu.emu_destroy(h)


def test_emulated_fused_steps_walsh15(oracle_mod, emu):
    """The fused key switch and rescale at the walsh15 shapes (N = 2^15: 16-column tiles of the
    7-bit column phase; 13 Q limbs, 4 P limbs, digits of 5, 5 and 3) with the row-phase
    geometry the device autotuner picks there (8 residues per thread, twiddles from the table):
    a rotation at the top level and at level 0, and a rescale, against the oracle."""
    O = oracle_mod
    prm = WALSH15
    N = 1 << prm["logN"]
    p, q = O.find_primes(prm["p_bits"], prm["q_bits"], N)
    o = O.OracleCtx(N, q, p, prm["dnum"])
    h = emu.emu_create(N, q, len(q), p, len(p), prm["dnum"])
    emu.emu_set_keyswitch_fusion(1)
    emu.emu_set_ntt_geometry(1)
    try:
        L = len(q)
        s = o.ternary(256, 3)
        rk = o.rotation_key(s, 512, 11)
        for level in (L - 1, 0):
            b, a = o.uniform(level + 1, 20 + level), o.uniform(level + 1, 40 + level)
            ob, oa = o.rotate(level, b, a, rk, 512)
            eb, ea = b.copy(), a.copy()
            emu.emu_keyswitch(h, level, a.copy(), rk, L - 1, eb, ea, 1, 0, o.galois(512))
            assert (eb == ob).all() and (ea == oa).all(), level
        x = o.uniform(L, 7)
        (ref,) = o.rescale(L - 1, [x])
        xs = x.copy()
        emu.emu_rescale(h, L - 1, xs)
        assert (xs[: (L - 1) * N] == ref).all()
    finally:
        emu.emu_set_keyswitch_fusion(0)
        emu.emu_set_ntt_geometry(0)
        emu.emu_destroy(h)


@pytest.mark.parametrize("logN", [10, 11, 12, 13, 14, 15, 16])
@pytest.mark.parametrize("geometry", [0, 1, 2, 3])
def test_emulated_ntt_geometries(oracle_mod, emu, logN, geometry):
    """Every NTT geometry the autotuner chooses from (8 or 16 residues per thread, twiddles
    staged or read from the table) on every supported ring degree (column / row phases of 5..8
    bits), against the oracle: lazy (36-bit) and fully reduced (61-bit) moduli."""
    O = oracle_mod
    N = 1 << logN
    p, q = O.find_primes([61], [36, 61], N)
    o = O.OracleCtx(N, q, p, 1)
    h = emu.emu_create(N, q, len(q), p, len(p), 1)
    emu.emu_set_ntt_geometry(geometry)
    try:
        x = o.uniform(len(q), 17)
        y = x.copy()
        emu.emu_ntt(h, y, len(q), 0, 0, 0)
        assert (y == o.ntt(x)).all()
        emu.emu_ntt(h, y, len(q), 0, 0, 1)
        assert (y == x).all()
    finally:
        emu.emu_set_ntt_geometry(0)
        emu.emu_destroy(h)


# NTT-friendly moduli of the walsh15 chain (36, 50 and 61 bits), the Mersenne prime 2^61 - 1 and
# the primes either side of 2^55 (where the Walsh sums switch from one word to 32-bit halves)
WIDE_MODULI = [68718428161, 1125899904679937, 2305843009208713217, 2305843009211596801, (1 << 61) - 1,
               36028797018963913, 36028797018963971]


def _bind_walsh(E):
    E.emu_reduce128.argtypes = [C.c_uint64, u64p, u64p, C.c_size_t, u64p]
    i8p = np.ctypeslib.ndpointer(dtype=np.int8, flags="C_CONTIGUOUS")
    E.emu_walsh_products.argtypes = [C.c_uint64, C.c_size_t, u64p, u64p, u64p, u64p, u64p, i8p, u64p, u64p]


@pytest.mark.parametrize("q", WIDE_MODULI)
def test_reduce128_canonical(emu, q):
    """reduce128 returns the canonical residue for any 128-bit value, including values a hair
    above or below a multiple of q, where a single-correction Barrett product can stay in [q, 2q)."""
    _bind_walsh(emu)
    rng = np.random.default_rng(q % 1000003)
    vals = [int(rng.integers(0, 1 << 63)) << 65 | int(rng.integers(0, 1 << 63)) for _ in range(4000)]
    top = ((1 << 128) - 1) // q
    for _ in range(4000):
        k = int(rng.integers(0, 1 << 62)) * (top >> 62) + int(rng.integers(0, 1 << 20))
        k = min(k, top)
        for d in (0, 1, 2, 7, q - 1, q - 3):
            v = k * q + d
            if v < (1 << 128):
                vals.append(v)
    vals += [(1 << 128) - 1, q * q - 1, q - 1, 0, q]
    hi = np.array([v >> 64 for v in vals], dtype=np.uint64)
    lo = np.array([v & ((1 << 64) - 1) for v in vals], dtype=np.uint64)
    out = np.zeros(len(vals), dtype=np.uint64)
    emu.emu_reduce128(q, hi, lo, len(vals), out)
    assert [int(x) for x in out] == [v % q for v in vals]


@pytest.mark.parametrize("q", WIDE_MODULI)
def test_mont_mul_exact(emu, q):
    """The Montgomery product is x y 2^-64 mod q, canonical, for x < 2q and y < q: random pairs and
    the pairs whose 128-bit product has a zero low word (x and y multiples of 2^32 or of higher
    powers of two, zero), where the carry out of the low words is the edge of the formula."""
    emu.emu_mont_mul.argtypes = [C.c_uint64, u64p, u64p, C.c_size_t, u64p]
    rng = np.random.default_rng(q % 999983)
    xs = [int(v) for v in rng.integers(0, 2 * q, 4000, dtype=np.uint64)]
    ys = [int(v) for v in rng.integers(0, q, 4000, dtype=np.uint64)]
    bits = q.bit_length() - 1
    for a in range(1, bits):
        for b in (64 - a, 65 - a, 70 - a):
            if 0 < b < bits:
                for ka, kb in ((1, 1), (3, 5), ((q >> a) - 1, (q >> b) - 1)):
                    if ka > 0 and kb > 0:
                        xs.append((ka << a) % (2 * q))
                        ys.append((kb << b) % q)
    xs += [0, 0, q - 1, 2 * q - 1, q, 1]
    ys += [0, q - 1, q - 1, q - 1, 1, 0]
    x = np.array(xs, dtype=np.uint64)
    y = np.array(ys, dtype=np.uint64)
    out = np.zeros(len(xs), dtype=np.uint64)
    emu.emu_mont_mul(q, x, y, len(xs), out)
    rinv = pow(1 << 64, -1, q)
    assert any((a * b) % (1 << 64) == 0 and a * b for a, b in zip(xs, ys))
    assert [int(v) for v in out] == [(a * b * rinv) % q for a, b in zip(xs, ys)]


def _walsh_model(q, lb, la, hb, ha, pt, coefs, c0):
    """The reference's sequence on exact integers: canonical low combinations (sums of added
    multiples), imaginary half times the encoded i, tensor products, products summed by mask."""
    def pair(s, hm, const):
        r = sum(int(coefs[0, hm, lm]) * s[lm] for lm in range(1, 16))
        im = sum(int(coefs[1, hm, lm]) * s[lm] for lm in range(1, 16))
        if const:
            r += int(c0[0, hm])
            im += int(c0[1, hm])
        return (r % q + (im % q) * pt) % q
    out = [pair(lb, 0, True), pair(la, 0, False)]
    rb = ra = rc = 0
    for hm in range(1, 16):
        x_b, x_a = pair(lb, hm, True), pair(la, hm, False)
        rb = (rb + x_b * hb[hm]) % q
        ra = (ra + x_a * hb[hm] + x_b * ha[hm]) % q
        rc = (rc + x_a * ha[hm]) % q
    return out + [rb, ra, rc]


@pytest.mark.parametrize("q", WIDE_MODULI)
def test_walsh_products_exact(emu, q):
    """The fused Walsh product body equals the reference's step-by-step modular sequence,
    with signs spread over [0, q) and bunched next to 0 and q, coefficients up to +-8."""
    _bind_walsh(emu)
    rng = np.random.default_rng(q % 999983)
    n = 48
    def draw(shape):
        v = rng.integers(0, q, size=shape, dtype=np.uint64)
        edge = rng.integers(0, 3, size=shape)
        small = rng.integers(0, 1 << 12, size=shape, dtype=np.uint64)
        v = np.where(edge == 1, small, v)
        v = np.where(edge == 2, np.uint64(q - 1) - small, v)
        return np.ascontiguousarray(v.astype(np.uint64))
    lb, la, hb, ha = (draw((n, 16)) for _ in range(4))
    pt = draw(n)
    coefs = rng.integers(-8, 9, size=(2, 16, 16)).astype(np.int8)
    coefs[:, :, 0] = 0
    coefs[0, 3, :] = 8
    coefs[1, 5, :] = -8
    c0 = rng.integers(0, q, size=(2, 16), dtype=np.uint64)
    out = np.zeros((n, 5), dtype=np.uint64)
    emu.emu_walsh_products(q, n, lb, la, hb, ha, pt, np.ascontiguousarray(coefs), np.ascontiguousarray(c0), out)
    for i in range(n):
        want = _walsh_model(q, [int(x) for x in lb[i]], [int(x) for x in la[i]], [int(x) for x in hb[i]],
                            [int(x) for x in ha[i]], int(pt[i]), coefs, c0)
        assert [int(x) for x in out[i]] == want, i


def test_staging_ring_never_overwrites_pending_uploads(emu):
    """The staging ring's placement, with every upload still pending (the host far ahead of the
    device, as in a long AES-CTR call): no region handed out may overlap an upload it did not wait
    for, also after early wraps put old uploads in front of newer ones."""
    emu.emu_ring_violations.restype = C.c_size_t
    emu.emu_ring_violations.argtypes = [C.c_uint64, C.c_size_t]
    for seed in (1, 2, 3):
        assert emu.emu_ring_violations(seed, 20000) == 0


def test_bundle_file_round_trip_and_damage(emu):
    """The key / plan bundle format (wg_bundle.hpp): random bundles survive encode and decode
    word for word; flipped bytes, truncations, a foreign magic and a newer version are all
    rejected."""
    emu.emu_bundle_roundtrip.restype = C.c_int
    emu.emu_bundle_roundtrip.argtypes = [C.c_uint64]
    emu.emu_bundle_damage_accepted.restype = C.c_size_t
    emu.emu_bundle_damage_accepted.argtypes = [C.c_uint64, C.c_size_t]
    for seed in range(5):
        assert emu.emu_bundle_roundtrip(seed) == 0
    assert emu.emu_bundle_damage_accepted(7, 500) == 0


def test_request_packing_is_first_fit(emu):
    """The batching service's packing (wg_batching.hpp): on seeded queues the taken requests are
    the first-fit choice in arrival order (oldest always taken, nothing skipped that fits) and
    the batch counts as full exactly when a request no longer fits or the slots are used up."""
    emu.emu_first_fit_violations.restype = C.c_size_t
    emu.emu_first_fit_violations.argtypes = [C.c_uint64, C.c_size_t]
    assert emu.emu_first_fit_violations(3, 20000) == 0
