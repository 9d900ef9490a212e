"""CPU emulation of the device kernels against the oracle.

tests/emu/wg_emulate.cpp compiles the product's kernel bodies (wg_ntt.cuh, wg_keyswitch.cuh)
and table builder with the host compiler and runs them thread by thread.  This checks index
logic, butterflies, HPS base changes and tables without a GPU; the GPU tests then check the
compiled kernels themselves.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from params import SMALL

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
    E.emu_keyswitch.argtypes = [C.c_void_p, C.c_size_t, u64p, u64p, C.c_size_t, u64p, u64p, C.c_int, C.c_int,
                                C.c_uint64]
    return E


@pytest.mark.parametrize("prm", SMALL)
def test_emulated_kernels_match_oracle(oracle_mod, emu, prm):
    O = oracle_mod
    N = 1 << prm["logN"]
    p, q = O.find_primes(prm["p_bits"], prm["q_bits"], N)
    o = O.OracleCtx(N, q, p, prm["dnum"])
    h = emu.emu_create(N, q, len(q), p, len(p), prm["dnum"])
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
    finally:
        emu.emu_destroy(h)


@pytest.mark.parametrize("logN", [13, 14, 15, 16])
def test_emulated_ntt_large_rings(oracle_mod, emu, logN):
    """Round plans of the larger rings (column / row phases of 6..8 bits)."""
    O = oracle_mod
    N = 1 << logN
    p, q = O.find_primes([61], [36, 61], N)
    o = O.OracleCtx(N, q, p, 1)
    h = emu.emu_create(N, q, len(q), p, len(p), 1)
    try:
        x = o.uniform(len(q), 17)
        y = x.copy()
        emu.emu_ntt(h, y, len(q), 0, 0, 0)
        assert (y == o.ntt(x)).all()
        emu.emu_ntt(h, y, len(q), 0, 0, 1)
        assert (y == x).all()
    finally:
        emu.emu_destroy(h)
