"""ctypes bindings for the CPU oracle (test infrastructure only).

Two libraries live here:

* ``_build/liboracle.so`` -- the plain-C restatement of the reference residue path
  (``ckks_oracle.c``), always buildable with gcc.
* ``_ref/libwalshref.so`` -- the reference itself, compiled from its own sources by
  ``make -C oracle ref`` with a thin harness (``ref_harness.cpp``).  Present only where the
  reference sources were available at build time.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libwalshref.so")

u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
i8p = np.ctypeslib.ndpointer(dtype=np.int8, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
szp = np.ctypeslib.ndpointer(dtype=np.uintp, flags="C_CONTIGUOUS")


# Where the reference project's sources are looked for: $REF_ROOT, else a checkout named
# `reference` beside this repository.  Only the build of the compiled reference reads them.
REF_ROOT = os.environ.get("REF_ROOT") or os.path.normpath(os.path.join(HERE, os.pardir, os.pardir, "reference"))


def build(ref: bool = False) -> None:
    """Compile the oracle (and, when asked and the sources exist, the reference harness)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref and os.path.isdir(REF_ROOT):
        subprocess.run(["make", "-s", "-j8", "-C", HERE, "ref"], check=True)


_lib = None
_ref = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        L.orc_find_primes.argtypes = [u64p, C.c_size_t, u64p, C.c_size_t, C.c_uint64, u64p, u64p]
        L.orc_ntt_tables.argtypes = [C.c_uint64, C.c_uint64, u64p, u64p, u64p, u64p, C.POINTER(C.c_uint64)]
        L.orc_ctx_create.restype = C.c_void_p
        L.orc_ctx_create.argtypes = [C.c_uint64, u64p, C.c_size_t, u64p, C.c_size_t, C.c_size_t]
        L.orc_ctx_destroy.argtypes = [C.c_void_p]
        L.orc_ctx_alpha.restype = C.c_size_t
        L.orc_ctx_alpha.argtypes = [C.c_void_p]
        L.orc_ntt.argtypes = [C.c_void_p, u64p, C.c_size_t, C.c_size_t, C.c_int, C.c_int, C.c_int]
        L.orc_keyswitch.argtypes = [C.c_void_p, C.c_size_t, u64p, u64p, C.c_size_t, u64p, u64p, C.c_int, C.c_int]
        L.orc_automorphism_map.argtypes = [C.c_uint64, C.c_uint64, u64p]
        L.orc_rotation_galois.restype = C.c_uint64
        L.orc_rotation_galois.argtypes = [C.c_uint64, C.c_int64]
        L.orc_rotate.argtypes = [C.c_void_p, C.c_size_t, u64p, u64p, u64p, C.c_size_t, C.c_int64]
        L.orc_conjugate.argtypes = [C.c_void_p, C.c_size_t, u64p, u64p, u64p, C.c_size_t]
        L.orc_mul.argtypes = [C.c_void_p, C.c_size_t, u64p, u64p, u64p, u64p, u64p]
        L.orc_relin.argtypes = [C.c_void_p, C.c_size_t, u64p, u64p, u64p, u64p, C.c_size_t]
        L.orc_rescale.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, u64p]
        L.orc_sample_ternary.argtypes = [C.c_uint64, C.c_size_t, C.c_uint64, i8p]
        L.orc_keygen_switch.argtypes = [C.c_void_p, i8p, C.c_int, i8p, C.c_double, C.c_uint64, u64p]
        L.orc_secret_automorphism.argtypes = [C.c_uint64, C.c_uint64, i8p, i8p]
        L.orc_uniform_poly.argtypes = [C.c_void_p, C.c_size_t, C.c_uint64, u64p]
        L.orc_encrypt.argtypes = [C.c_void_p, C.c_size_t, u64p, i8p, C.c_double, C.c_uint64, u64p, u64p]
        L.orc_decrypt_coeffs.argtypes = [C.c_void_p, C.c_size_t, u64p, u64p, i8p, f64p]
        L.orc_barrett_mul.restype = C.c_uint64
        L.orc_barrett_mul.argtypes = [C.c_uint64] * 5
        L.orc_lt_stage.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, u64p, u64p, C.c_size_t, C.c_size_t, C.c_int,
                                   C.c_void_p, i64p, C.c_size_t, C.c_size_t, u64p, u64p]
        L.orc_batched_ops.argtypes = [C.c_void_p, C.c_size_t, szp, u64p, u64p, u64p, u64p, u64p,
                                      C.c_void_p, i64p, C.c_size_t, C.c_size_t, C.c_int]
        L.orc_modraise.argtypes = [C.c_void_p, C.c_size_t, u64p, u64p]
        L.orc_q0p0_switch.argtypes = [C.c_void_p, u64p, u64p, u64p]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        R = C.CDLL(REF_SO)
        R.ref_last_error.restype = C.c_char_p
        R.ref_find_primes.argtypes = [u64p, C.c_size_t, u64p, C.c_size_t, C.c_uint64, u64p, u64p]
        R.ref_ntt_tables.argtypes = [C.c_uint64, C.c_uint64, u64p, u64p, u64p, u64p, C.POINTER(C.c_uint64), u64p]
        R.ref_ctx_create.restype = C.c_void_p
        R.ref_ctx_create.argtypes = [C.c_uint64, u64p, C.c_size_t, u64p, C.c_size_t, C.c_size_t, C.c_size_t,
                                     C.c_double, C.c_double, i64p, C.c_size_t]
        R.ref_ctx_destroy.argtypes = [C.c_void_p]
        R.ref_ctx_moduli.argtypes = [C.c_void_p, u64p, C.POINTER(C.c_size_t), u64p, C.POINTER(C.c_size_t)]
        R.ref_ctx_ntt.argtypes = [C.c_void_p, u64p, C.c_size_t, C.c_int, C.c_int]
        R.ref_ctx_key_shape.argtypes = [C.c_void_p, C.c_int, C.c_int64, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]
        R.ref_ctx_key.argtypes = [C.c_void_p, C.c_int, C.c_int64, u64p]
        R.ref_ctx_map.argtypes = [C.c_void_p, C.c_int, C.c_int64, u64p]
        R.ref_ctx_secret.argtypes = [C.c_void_p, u64p]
        R.ref_keyswitch.argtypes = [C.c_void_p, C.c_size_t, u64p, u64p, C.c_size_t, C.c_size_t, u64p, u64p,
                                    C.c_int, C.c_int, C.c_int]
        R.ref_rotate.argtypes = [C.c_void_p, C.c_size_t, u64p, u64p, C.c_int64]
        R.ref_conjugate.argtypes = [C.c_void_p, C.c_size_t, u64p, u64p]
        R.ref_mul.argtypes = [C.c_void_p, C.c_size_t, u64p, u64p, u64p, u64p, u64p]
        R.ref_relin.argtypes = [C.c_void_p, C.c_size_t, u64p, u64p, u64p]
        R.ref_rescale.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, u64p]
        R.ref_hoisted_rotations.argtypes = [C.c_void_p, C.c_size_t, u64p, u64p, i64p, C.c_size_t, u64p]
        R.ref_batched_ops.argtypes = [C.c_void_p, C.c_size_t, szp, u64p, u64p, u64p, u64p, i64p, C.c_size_t,
                                      C.c_int, C.POINTER(C.c_double)]
        R.ref_max_threads.restype = C.c_int
        _ref = R
    return _ref


def _check(rc: int, who: str) -> None:
    if rc != 0:
        msg = ref().ref_last_error().decode() if who.startswith("ref") else ""
        raise RuntimeError(f"{who} failed ({rc}) {msg}")


# ------------------------------------------------------------------------------------------
# Parameter helpers
# ------------------------------------------------------------------------------------------
def find_primes(p_bits, q_bits, N):
    pb = np.ascontiguousarray(p_bits, dtype=np.uint64)
    qb = np.ascontiguousarray(q_bits, dtype=np.uint64)
    p = np.zeros(len(pb), np.uint64)
    q = np.zeros(len(qb), np.uint64)
    _check(lib().orc_find_primes(pb, len(pb), qb, len(qb), N, p, q), "orc_find_primes")
    return p, q


def ntt_tables(N, q):
    f = np.zeros(N, np.uint64)
    fs = np.zeros(N, np.uint64)
    i = np.zeros(N, np.uint64)
    is_ = np.zeros(N + 1, np.uint64)
    ninv = C.c_uint64()
    _check(lib().orc_ntt_tables(N, int(q), f, fs, i, is_, C.byref(ninv)), "orc_ntt_tables")
    return f, fs, i, is_, ninv.value


class OracleCtx:
    """Oracle context for one parameter set (moduli Q, P, dnum)."""

    def __init__(self, N, q, p, dnum):
        self.N = int(N)
        self.q = np.ascontiguousarray(q, dtype=np.uint64)
        self.p = np.ascontiguousarray(p, dtype=np.uint64)
        self.dnum = int(dnum)
        self.h = lib().orc_ctx_create(self.N, self.q, len(self.q), self.p, len(self.p), self.dnum)
        if not self.h:
            raise ValueError("invalid oracle parameters")
        self.alpha = lib().orc_ctx_alpha(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_ctx_destroy(self.h)
            self.h = None

    @property
    def nq(self):
        return len(self.q)

    @property
    def np_(self):
        return len(self.p)

    def parts(self, level):
        return min(self.dnum, (level + 1 + self.alpha - 1) // self.alpha)

    def key_size(self, key_level=None):
        kl = self.nq - 1 if key_level is None else key_level
        return self.dnum_top() * 2 * (kl + 1 + self.np_) * self.N

    def dnum_top(self):
        return self.parts(self.nq - 1)

    def ntt(self, poly, first=0, which=0, inverse=False, lazy=False):
        poly = np.ascontiguousarray(poly, dtype=np.uint64).copy()
        limbs = poly.size // self.N
        lib().orc_ntt(self.h, poly, first, limbs, int(which), int(inverse), int(lazy))
        return poly

    def uniform(self, limbs, seed):
        out = np.zeros(limbs * self.N, np.uint64)
        lib().orc_uniform_poly(self.h, limbs, seed, out)
        return out

    def ternary(self, h, seed):
        s = np.zeros(self.N, np.int8)
        lib().orc_sample_ternary(self.N, h, seed, s)
        return s

    def keygen(self, src, dst, seed, square=False, sigma=3.2):
        key = np.zeros(self.key_size(), np.uint64)
        _check(lib().orc_keygen_switch(self.h, src, int(square), dst, sigma, seed, key), "orc_keygen")
        return key

    def rotation_key(self, s, rotation, seed):
        g_inv = lib().orc_rotation_galois(self.N, -rotation)
        sd = np.zeros(self.N, np.int8)
        lib().orc_secret_automorphism(self.N, g_inv, s, sd)
        return self.keygen(s, sd, seed)

    def conjugation_key(self, s, seed):
        sd = np.zeros(self.N, np.int8)
        lib().orc_secret_automorphism(self.N, 2 * self.N - 1, s, sd)
        return self.keygen(sd, s, seed)

    def relin_key(self, s, seed):
        return self.keygen(s, s, seed, square=True)

    def keyswitch(self, level, key_term, key, b, a, b_add=True, a_add=False, key_level=None):
        kl = self.nq - 1 if key_level is None else key_level
        b = np.ascontiguousarray(b, dtype=np.uint64).copy()
        a = np.ascontiguousarray(a, dtype=np.uint64).copy()
        kt = np.ascontiguousarray(key_term, dtype=np.uint64)
        _check(lib().orc_keyswitch(self.h, level, kt, np.ascontiguousarray(key), kl, b, a,
                                   int(b_add), int(a_add)), "orc_keyswitch")
        return b, a

    def rotate(self, level, b, a, key, rotation, key_level=None):
        kl = self.nq - 1 if key_level is None else key_level
        b = np.ascontiguousarray(b, dtype=np.uint64).copy()
        a = np.ascontiguousarray(a, dtype=np.uint64).copy()
        _check(lib().orc_rotate(self.h, level, b, a, np.ascontiguousarray(key), kl, rotation), "orc_rotate")
        return b, a

    def modraise(self, target_level, b, a):
        """Limb 0 of (b, a) raised to target_level+1 limbs (ModRaise)."""
        n = (target_level + 1) * self.N
        bo = np.zeros(n, np.uint64)
        ao = np.zeros(n, np.uint64)
        bo[: self.N] = np.asarray(b, dtype=np.uint64)[: self.N]
        ao[: self.N] = np.asarray(a, dtype=np.uint64)[: self.N]
        _check(lib().orc_modraise(self.h, target_level, bo, ao), "orc_modraise")
        return bo, ao

    def q0p0_switch(self, key, b, a):
        """Level-0 dense-to-sparse switch with the compact q0/p0 key."""
        b = np.ascontiguousarray(b[: self.N], dtype=np.uint64).copy()
        a = np.ascontiguousarray(a[: self.N], dtype=np.uint64).copy()
        _check(lib().orc_q0p0_switch(self.h, np.ascontiguousarray(key, dtype=np.uint64), b, a), "orc_q0p0_switch")
        return b, a

    def conjugate(self, level, b, a, key, key_level=None):
        kl = self.nq - 1 if key_level is None else key_level
        b = np.ascontiguousarray(b, dtype=np.uint64).copy()
        a = np.ascontiguousarray(a, dtype=np.uint64).copy()
        _check(lib().orc_conjugate(self.h, level, b, a, np.ascontiguousarray(key), kl), "orc_conjugate")
        return b, a

    def mul(self, level, b1, a1, b2, a2):
        b1 = np.ascontiguousarray(b1, dtype=np.uint64).copy()
        a1 = np.ascontiguousarray(a1, dtype=np.uint64).copy()
        c2 = np.zeros_like(b1)
        _check(lib().orc_mul(self.h, level, b1, a1, np.ascontiguousarray(b2), np.ascontiguousarray(a2), c2),
               "orc_mul")
        return b1, a1, c2

    def relin(self, level, c0, c1, c2, key, key_level=None):
        kl = self.nq - 1 if key_level is None else key_level
        c0 = np.ascontiguousarray(c0, dtype=np.uint64).copy()
        c1 = np.ascontiguousarray(c1, dtype=np.uint64).copy()
        _check(lib().orc_relin(self.h, level, c0, c1, np.ascontiguousarray(c2), np.ascontiguousarray(key), kl),
               "orc_relin")
        return c0, c1

    def rescale(self, level, polys):
        """polys: list of (level+1)*N arrays; returns list of level*N arrays."""
        n = (level + 1) * self.N
        flat = np.concatenate([np.ascontiguousarray(p, dtype=np.uint64) for p in polys])
        _check(lib().orc_rescale(self.h, level, len(polys), flat), "orc_rescale")
        return [flat[k * n:k * n + level * self.N].copy() for k in range(len(polys))]

    def automorphism_map(self, g):
        m = np.zeros(self.N, np.uint64)
        lib().orc_automorphism_map(self.N, g, m)
        return m

    def galois(self, rotation):
        return lib().orc_rotation_galois(self.N, rotation)

    def encrypt(self, level, m_ntt, s, seed, sigma=3.2):
        n = (level + 1) * self.N
        b = np.zeros(n, np.uint64)
        a = np.zeros(n, np.uint64)
        _check(lib().orc_encrypt(self.h, level, np.ascontiguousarray(m_ntt, dtype=np.uint64), s, sigma, seed, b, a),
               "orc_encrypt")
        return b, a

    def decrypt_coeffs(self, level, b, a, s):
        out = np.zeros(self.N, np.float64)
        _check(lib().orc_decrypt_coeffs(self.h, level, np.ascontiguousarray(b), np.ascontiguousarray(a), s, out),
               "orc_decrypt")
        return out

    def lt_stage(self, level, indices, diags, baby, slots, rescale, keys, b, a, key_level=None):
        """keys: dict rotation -> flat key array."""
        kl = self.nq - 1 if key_level is None else key_level
        rots = np.ascontiguousarray(list(keys.keys()), dtype=np.int64)
        arrs = [np.ascontiguousarray(keys[int(r)], dtype=np.uint64) for r in rots]
        ptrs = (C.c_void_p * len(arrs))(*[x.ctypes.data for x in arrs])
        b = np.ascontiguousarray(b, dtype=np.uint64).copy()
        a = np.ascontiguousarray(a, dtype=np.uint64).copy()
        _check(lib().orc_lt_stage(self.h, level, len(indices), np.ascontiguousarray(indices, dtype=np.uint64),
                                  np.ascontiguousarray(diags, dtype=np.uint64), baby, slots, int(rescale),
                                  C.cast(ptrs, C.c_void_p), rots, len(rots), kl, b, a), "orc_lt_stage")
        n = (level if rescale else level + 1) * self.N
        return b[:n], a[:n]

    def batched_ops(self, levels, x_b, x_a, y_b, y_a, relin_key, rot_keys, rots, stride, threads):
        """CPU timing baseline: x_* updated in place.  rot_keys: list of key arrays."""
        levels = np.ascontiguousarray(levels, dtype=np.uintp)
        ptrs = (C.c_void_p * len(rot_keys))(*[k.ctypes.data for k in rot_keys])
        rc = lib().orc_batched_ops(self.h, len(levels), levels, x_b, x_a, y_b, y_a, relin_key,
                                   C.cast(ptrs, C.c_void_p), np.ascontiguousarray(rots, dtype=np.int64),
                                   self.nq - 1, stride, threads)
        _check(rc, "orc_batched_ops")


def _secret_from_ntt(h, N, nq, low=False):
    """A context's ternary secret (or its bootstrapping sparse secret) as N int8 coefficients:
    the inverse NTT of limb 0 of its NTT form."""
    R = ref()
    R.ref_ctx_low_secret.argtypes = [C.c_void_p, u64p]
    R.ref_ctx_ntt.argtypes = [C.c_void_p, u64p, C.c_size_t, C.c_int, C.c_int]
    sk = np.zeros(nq * N, np.uint64)
    _check((R.ref_ctx_low_secret if low else R.ref_ctx_secret)(h, sk), "ref_ctx_secret")
    c0 = np.ascontiguousarray(sk[:N]).copy()
    _check(R.ref_ctx_ntt(h, c0, 1, 1, 0), "ref_ctx_ntt")
    q0 = None
    vals = c0.tolist()
    out = np.zeros(N, np.int8)
    big = max(vals)
    for i, v in enumerate(vals):
        if v == 0:
            continue
        if v == 1:
            out[i] = 1
        elif v == big:  # q0 - 1
            out[i] = -1
        else:
            return q0
    return out


class RefCtx:
    """The reference's own CKKSContext (custom moduli schedule, no bootstrapping keys)."""

    def __init__(self, N, q_bits, p_bits, dnum, h=192, sigma=3.2, scale=2.0 ** 40, rotations=(1,)):
        R = ref()
        qb = np.ascontiguousarray(q_bits, dtype=np.uint64)
        pb = np.ascontiguousarray(p_bits, dtype=np.uint64)
        rots = np.ascontiguousarray(rotations, dtype=np.int64)
        self.N = int(N)
        self.h = R.ref_ctx_create(self.N, qb, len(qb), pb, len(pb), dnum, h, sigma, scale, rots, len(rots))
        if not self.h:
            raise RuntimeError("ref_ctx_create: " + R.ref_last_error().decode())
        nq, np_ = C.c_size_t(), C.c_size_t()
        _check(R.ref_ctx_moduli(self.h, np.zeros(64, np.uint64), C.byref(nq), np.zeros(64, np.uint64),
                                C.byref(np_)), "ref_ctx_moduli")
        self.q = np.zeros(nq.value, np.uint64)
        self.p = np.zeros(np_.value, np.uint64)
        _check(R.ref_ctx_moduli(self.h, self.q, C.byref(nq), self.p, C.byref(np_)), "ref_ctx_moduli")
        self.dnum = dnum

    def __del__(self):
        if getattr(self, "h", None):
            ref().ref_ctx_destroy(self.h)
            self.h = None

    def ntt(self, poly, inverse=False, lazy=False):
        poly = np.ascontiguousarray(poly, dtype=np.uint64).copy()
        _check(ref().ref_ctx_ntt(self.h, poly, poly.size // self.N, int(inverse), int(lazy)), "ref_ctx_ntt")
        return poly

    def key(self, kind, rot=0):
        parts, kl = C.c_size_t(), C.c_size_t()
        _check(ref().ref_ctx_key_shape(self.h, kind, rot, C.byref(parts), C.byref(kl)), "ref_ctx_key_shape")
        size = parts.value * 2 * (kl.value + 1 + len(self.p)) * self.N
        out = np.zeros(size, np.uint64)
        _check(ref().ref_ctx_key(self.h, kind, rot, out), "ref_ctx_key")
        return out, parts.value, kl.value

    def map(self, kind, rot=0):
        out = np.zeros(self.N, np.uint64)
        _check(ref().ref_ctx_map(self.h, kind, rot, out), "ref_ctx_map")
        return out

    def keyswitch(self, level, key_term, key, parts, key_level, b, a, b_add=True, a_add=False):
        b = np.ascontiguousarray(b, dtype=np.uint64).copy()
        a = np.ascontiguousarray(a, dtype=np.uint64).copy()
        kt = np.ascontiguousarray(key_term, dtype=np.uint64).copy()
        _check(ref().ref_keyswitch(self.h, level, kt, np.ascontiguousarray(key), parts, key_level, b, a,
                                   int(b_add), int(a_add), 1), "ref_keyswitch")
        return b, a

    def batched_ops_seconds(self, levels, x_b, x_a, y_b, y_a, rots, stride, threads):
        """Wall time of the reference's mul + relin + rescale + rotate on every ciphertext i at
        levels[i] (buffers of `stride` words per ciphertext, x updated in place), OpenMP over
        ciphertexts on `threads` threads (ref_batched_ops)."""
        sec = C.c_double()
        _check(ref().ref_batched_ops(self.h, len(levels), np.ascontiguousarray(levels, np.uintp), x_b, x_a, y_b, y_a,
                                     np.ascontiguousarray(rots, np.int64), stride, int(threads), C.byref(sec)),
               "ref_batched_ops")
        return sec.value

    def rotate(self, level, b, a, rot):
        b = np.ascontiguousarray(b, dtype=np.uint64).copy()
        a = np.ascontiguousarray(a, dtype=np.uint64).copy()
        _check(ref().ref_rotate(self.h, level, b, a, rot), "ref_rotate")
        return b, a

    def conjugate(self, level, b, a):
        b = np.ascontiguousarray(b, dtype=np.uint64).copy()
        a = np.ascontiguousarray(a, dtype=np.uint64).copy()
        _check(ref().ref_conjugate(self.h, level, b, a), "ref_conjugate")
        return b, a

    def mul(self, level, b1, a1, b2, a2):
        b1 = np.ascontiguousarray(b1, dtype=np.uint64).copy()
        a1 = np.ascontiguousarray(a1, dtype=np.uint64).copy()
        c2 = np.zeros_like(b1)
        _check(ref().ref_mul(self.h, level, b1, a1, np.ascontiguousarray(b2), np.ascontiguousarray(a2), c2),
               "ref_mul")
        return b1, a1, c2

    def relin(self, level, c0, c1, c2):
        c0 = np.ascontiguousarray(c0, dtype=np.uint64).copy()
        c1 = np.ascontiguousarray(c1, dtype=np.uint64).copy()
        _check(ref().ref_relin(self.h, level, c0, c1, np.ascontiguousarray(c2)), "ref_relin")
        return c0, c1

    def rescale(self, level, polys):
        n = (level + 1) * self.N
        flat = np.concatenate([np.ascontiguousarray(p, dtype=np.uint64) for p in polys])
        _check(ref().ref_rescale(self.h, level, len(polys), flat), "ref_rescale")
        return [flat[k * n:k * n + level * self.N].copy() for k in range(len(polys))]

    def secret_coeffs(self):
        """The context's ternary secret as N int8 coefficients (inverse NTT of its limb 0)."""
        return _secret_from_ntt(self.h, self.N, len(self.q))

    def encrypt_from_parts(self, level, pt, secret, a, e):
        """ckks_encrypt_custom_eval of the evaluation-form plaintext pt with the mask a and noise e
        given (ref_encrypt_from_parts): (b, a)."""
        R = ref()
        R.ref_encrypt_from_parts.argtypes = [C.c_void_p, C.c_size_t, u64p,
                                             np.ctypeslib.ndpointer(dtype=np.int8, flags="C_CONTIGUOUS"), u64p,
                                             np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS"), u64p,
                                             u64p]
        n = (level + 1) * self.N
        ob, oa = np.zeros(n, np.uint64), np.zeros(n, np.uint64)
        _check(R.ref_encrypt_from_parts(self.h, level, np.ascontiguousarray(pt[:n], np.uint64),
                                        np.ascontiguousarray(secret, np.int8), np.ascontiguousarray(a[:n], np.uint64),
                                        np.ascontiguousarray(e, np.int64), ob, oa), "ref_encrypt_from_parts")
        return ob, oa

    def switch_key_from_parts(self, kind, rotation, secret, a, e, target=None):
        """The reference's rotation (kind 0) / conjugation (kind 1) / relinearisation (kind 2) /
        dense-to-sparse (kind 3, compact q0 p0) / sparse-to-dense (kind 4) key construction (secret
        switches from `secret` to `target`) with the mask
        a and noise e given (ref_switch_key_from_parts): flat [part][a|b][limbs][N]."""
        R = ref()
        i8p = np.ctypeslib.ndpointer(dtype=np.int8, flags="C_CONTIGUOUS")
        R.ref_switch_key_from_parts.argtypes = [C.c_void_p, C.c_int, C.c_int64, i8p, i8p, u64p,
                                                np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS"), u64p]
        a = np.ascontiguousarray(a, dtype=np.uint64)
        out = np.zeros(2 * a.size, np.uint64)
        tgt = np.ascontiguousarray(secret if target is None else target, dtype=np.int8)
        _check(R.ref_switch_key_from_parts(self.h, int(kind), int(rotation),
                                                 np.ascontiguousarray(secret, dtype=np.int8), tgt, a,
                                                 np.ascontiguousarray(e, dtype=np.int64), out),
               "ref_switch_key_from_parts")
        return out

    def hoisted_rotations(self, level, b, a, rots):
        n = (level + 1) * self.N
        out = np.zeros(len(rots) * 2 * n, np.uint64)
        _check(ref().ref_hoisted_rotations(self.h, level, np.ascontiguousarray(b), np.ascontiguousarray(a),
                                           np.ascontiguousarray(rots, dtype=np.int64), len(rots), out),
               "ref_hoisted_rotations")
        return out.reshape(len(rots), 2, n)


class RefXboot(RefCtx):
    """The reference's XBOOT chain at N = 2^15 (AESXBoot15Config without bootstrapping: 17 Q limbs,
    5 P limbs, dnum 5) and the XBOOT S-box restated on its public operations
    (ref_xboot_sbox, following src/ckks/operations/circuits/aes/ckks_aes_ctr.cpp:160-336)."""

    def __init__(self):
        R = ref()
        R.ref_xboot15_create.restype = C.c_void_p
        R.ref_xboot_sbox.argtypes = [C.c_void_p, C.c_size_t, C.c_double, u64p, u64p, szp, f64p]
        R.ref_xboot_sbox_coefficients.argtypes = [np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")]
        self.h = R.ref_xboot15_create()
        if not self.h:
            raise RuntimeError("ref_xboot15_create: " + R.ref_last_error().decode())
        self.N = 1 << 15
        nq, np_ = C.c_size_t(), C.c_size_t()
        _check(R.ref_ctx_moduli(self.h, np.zeros(64, np.uint64), C.byref(nq), np.zeros(64, np.uint64),
                                C.byref(np_)), "ref_ctx_moduli")
        self.q = np.zeros(nq.value, np.uint64)
        self.p = np.zeros(np_.value, np.uint64)
        _check(R.ref_ctx_moduli(self.h, self.q, C.byref(nq), self.p, C.byref(np_)), "ref_ctx_moduli")
        self.dnum = 5

    def sbox(self, level, scale, bits):
        """The XBOOT S-box on 8 bit ciphertexts [(b, a)] at `level`: [(b, a, level, scale)] x 8."""
        n = (level + 1) * self.N
        flat = np.concatenate([np.concatenate([np.asarray(b[:n], np.uint64), np.asarray(a[:n], np.uint64)])
                               for b, a in bits])
        out = np.zeros(16 * len(self.q) * self.N, np.uint64)
        lv = np.zeros(8, np.uintp)
        sc = np.zeros(8, np.float64)
        _check(ref().ref_xboot_sbox(self.h, level, float(scale), flat, out, lv, sc), "ref_xboot_sbox")
        res, off = [], 0
        for k in range(8):
            m = (int(lv[k]) + 1) * self.N
            res.append((out[off:off + m].copy(), out[off + m:off + 2 * m].copy(), int(lv[k]), float(sc[k])))
            off += 2 * m
        return res

    def sbox_layer_seconds(self, level, scale, bits, instances, threads=0):
        """Wall time of `instances` XBOOT S-boxes on copies of the 8 bit ciphertexts `bits`, run as
        the reference's sub_bytes_inplace runs its byte positions (OpenMP dynamic over instances,
        src/ckks/operations/circuits/aes/ckks_aes_ctr.cpp:474-509) on `threads` threads (0: the
        OpenMP default).  The outputs are discarded."""
        R = ref()
        R.ref_xboot_sbox_layer.argtypes = [C.c_void_p, C.c_size_t, C.c_double, u64p, C.c_size_t, C.c_int,
                                           C.POINTER(C.c_double)]
        n = (level + 1) * self.N
        flat = np.concatenate([np.concatenate([np.asarray(b[:n], np.uint64), np.asarray(a[:n], np.uint64)])
                               for b, a in bits])
        sec = C.c_double()
        _check(R.ref_xboot_sbox_layer(self.h, level, float(scale), flat, instances, threads, C.byref(sec)),
               "ref_xboot_sbox_layer")
        return sec.value

    @staticmethod
    def coefficients():
        out = np.zeros(8 * 256, np.int64)
        ref().ref_xboot_sbox_coefficients.argtypes = [np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")]
        _check(ref().ref_xboot_sbox_coefficients(out), "ref_xboot_sbox_coefficients")
        return out.reshape(8, 256)


class RefPlans:
    """The reference's S2C / C2S plans and rotation keys of a bootstrapping parameter set:
    walsh15 (ref_walsh15_plans_create, or ref_walsh15_bts_create with bootstrap_keys), or the
    XBOOT sets with their bootstrapping keys (preset "xboot15" / "xboot15-sparse",
    ref_xboot15_bts_create; "xboot14" / "xboot14-sparse", ref_xboot14_bts_create)."""

    def __init__(self, bootstrap_keys=False, preset="walsh15"):
        R = ref()
        R.ref_walsh15_plans_create.restype = C.c_void_p
        R.ref_walsh15_bts_create.restype = C.c_void_p
        R.ref_xboot15_bts_create.restype = C.c_void_p
        R.ref_xboot15_bts_create.argtypes = [C.c_int]
        R.ref_xboot14_bts_create.restype = C.c_void_p
        R.ref_xboot14_bts_create.argtypes = [C.c_int]
        R.ref_bootstrap_pair.argtypes = [C.c_void_p, C.c_size_t, C.c_double, C.c_double] + [u64p] * 8 + \
            [C.POINTER(C.c_size_t), C.POINTER(C.c_double)]
        R.ref_xboot_key_bits.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t, u64p, f64p, szp]
        R.ref_ctx_key_words.argtypes = [C.c_void_p, C.c_int, C.c_int64, C.POINTER(C.c_size_t)]
        R.ref_modraise.argtypes = [C.c_void_p, C.c_size_t, u64p, u64p]
        R.ref_dense_to_sparse.argtypes = [C.c_void_p, u64p, u64p]
        R.ref_sparse_to_dense.argtypes = [C.c_void_p, C.c_size_t, u64p, u64p]
        R.ref_ctx_scale.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        R.ref_build_scaled_s2c.argtypes = [C.c_void_p, C.c_uint64]
        R.ref_aes_key_bits.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t, u64p, f64p, C.POINTER(C.c_size_t)]
        R.ref_aes_ctr.argtypes = [C.c_void_p, u64p, f64p, C.c_size_t, C.c_char_p, C.c_char_p, C.c_size_t, u64p, szp,
                                  f64p]
        R.ref_decrypt.argtypes = [C.c_void_p, C.c_size_t, C.c_double, u64p, u64p, f64p, f64p]
        R.ref_encode.argtypes = [C.c_void_p, f64p, f64p, C.c_double, C.c_size_t, u64p]
        R.ref_walsh_sbox.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_double, u64p, u64p, szp, f64p]
        R.ref_walsh_sbox_layer.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_double, u64p, C.c_size_t, C.c_int,
                                           C.POINTER(C.c_double)]
        R.ref_bts_info.argtypes = [C.c_void_p] + [C.POINTER(C.c_size_t)] * 6 + [C.POINTER(C.c_double),
                                                                               C.POINTER(C.c_size_t)]
        R.ref_bts_evalmod_coeffs.argtypes = [C.c_void_p, f64p]
        R.ref_bootstrap_evalmod.argtypes = [C.c_void_p, C.c_size_t, C.c_double, u64p, u64p, u64p, u64p, u64p, u64p,
                                            C.POINTER(C.c_size_t), C.POINTER(C.c_double)]
        R.ref_evalchebyshev.argtypes = [C.c_void_p, C.c_size_t, C.c_double, f64p, C.c_size_t, C.c_double, u64p, u64p,
                                        C.POINTER(C.c_size_t), C.POINTER(C.c_double), u64p, u64p]
        R.ref_plan_stage_count.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_size_t), C.POINTER(C.c_int)]
        R.ref_plan_stage_info.argtypes = [C.c_void_p, C.c_int, C.c_size_t] + [C.POINTER(C.c_size_t)] * 2 + \
            [C.POINTER(C.c_int), C.POINTER(C.c_size_t), C.POINTER(C.c_int), C.POINTER(C.c_size_t)]
        R.ref_plan_stage_data.argtypes = [C.c_void_p, C.c_int, C.c_size_t, u64p, C.c_void_p]
        R.ref_lt_stage.argtypes = [C.c_void_p, C.c_int, C.c_size_t, C.c_size_t, u64p, u64p, u64p, u64p,
                                   C.POINTER(C.c_size_t)]
        R.ref_ctx_rotations.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_size_t)]
        if preset == "walsh15":
            self.h = R.ref_walsh15_bts_create() if bootstrap_keys else R.ref_walsh15_plans_create()
            self.dnum = 3
        elif preset in ("xboot15", "xboot15-sparse"):
            self.h = R.ref_xboot15_bts_create(1 if preset == "xboot15-sparse" else 0)
            self.dnum = 5
        elif preset in ("xboot14", "xboot14-sparse"):
            self.h = R.ref_xboot14_bts_create(1 if preset == "xboot14-sparse" else 0)
            self.dnum = 13
        else:
            raise ValueError(f"unknown parameter preset {preset!r}")
        if not self.h:
            raise RuntimeError(f"ref {preset} context: " + R.ref_last_error().decode())
        self.preset = preset
        nq, np_ = C.c_size_t(), C.c_size_t()
        _check(R.ref_ctx_moduli(self.h, np.zeros(64, np.uint64), C.byref(nq), np.zeros(64, np.uint64), C.byref(np_)),
               "ref_ctx_moduli")
        self.q = np.zeros(nq.value, np.uint64)
        self.p = np.zeros(np_.value, np.uint64)
        _check(R.ref_ctx_moduli(self.h, self.q, C.byref(nq), self.p, C.byref(np_)), "ref_ctx_moduli")
        self.N = 1 << (14 if preset.startswith("xboot14") else 15)
        sc = C.c_double()
        _check(R.ref_ctx_scale(self.h, C.byref(sc)), "ref_ctx_scale")
        self.scale = sc.value

    def __del__(self):
        if getattr(self, "h", None):
            ref().ref_ctx_destroy(self.h)
            self.h = None

    def stages(self, which):
        n, qp = C.c_size_t(), C.c_int()
        _check(ref().ref_plan_stage_count(self.h, which, C.byref(n), C.byref(qp)), "ref_plan_stage_count")
        return n.value

    def stage(self, which, stage, with_diagonals=True):
        nt, baby, qpl, slots = C.c_size_t(), C.c_size_t(), C.c_size_t(), C.c_size_t()
        resc, mont = C.c_int(), C.c_int()
        _check(ref().ref_plan_stage_info(self.h, which, stage, C.byref(nt), C.byref(baby), C.byref(resc),
                                         C.byref(qpl), C.byref(mont), C.byref(slots)), "ref_plan_stage_info")
        idx = np.zeros(nt.value, np.uint64)
        diags = np.zeros(nt.value * qpl.value * self.N, np.uint64) if with_diagonals else None
        _check(ref().ref_plan_stage_data(self.h, which, stage, idx, diags.ctypes.data if with_diagonals else None),
               "ref_plan_stage_data")
        return dict(nterms=nt.value, baby=baby.value, rescale=bool(resc.value), qp_limbs=qpl.value,
                    montgomery=bool(mont.value), slot_count=slots.value, indices=idx, diagonals=diags)

    def plan_seconds(self, which, level, b, a, count, threads=0):
        """Wall time of the whole plan `which` (0: SlotToCoeff, 1: CoeffToSlot; every stage in
        order through ckks_apply_linear_transform_owned_stage_qp) on `count` copies of (b, a) at
        `level`, OpenMP over ciphertexts on `threads` threads (ref_lt_plan_seconds)."""
        R = ref()
        R.ref_lt_plan_seconds.argtypes = [C.c_void_p, C.c_int, C.c_size_t, u64p, u64p, C.c_size_t, C.c_int,
                                          C.POINTER(C.c_double)]
        n = (level + 1) * self.N
        sec = C.c_double()
        _check(R.ref_lt_plan_seconds(self.h, which, level, np.ascontiguousarray(b[:n], np.uint64),
                                     np.ascontiguousarray(a[:n], np.uint64), count, threads, C.byref(sec)),
               "ref_lt_plan_seconds")
        return sec.value

    def apply_stage(self, which, stage, level, b, a):
        n = (level + 1) * self.N
        ob = np.zeros(n, np.uint64)
        oa = np.zeros(n, np.uint64)
        lv = C.c_size_t()
        _check(ref().ref_lt_stage(self.h, which, stage, level, np.ascontiguousarray(b), np.ascontiguousarray(a),
                                  ob, oa, C.byref(lv)), "ref_lt_stage")
        return ob[:(lv.value + 1) * self.N], oa[:(lv.value + 1) * self.N], lv.value

    def rotations(self):
        n = C.c_size_t()
        _check(ref().ref_ctx_rotations(self.h, None, C.byref(n)), "ref_ctx_rotations")
        out = np.zeros(n.value, np.int64)
        _check(ref().ref_ctx_rotations(self.h, out.ctypes.data, C.byref(n)), "ref_ctx_rotations")
        return out

    def key(self, rot, kind=0):
        """Switching key as stored: (flat [part][a|b][limbs][N], parts, key level).  kind 0
        rotation, 1 conjugation, 2 relinearization, 3 dense-to-sparse (compact q0/p0 key),
        4 sparse-to-dense."""
        parts, kl, words = C.c_size_t(), C.c_size_t(), C.c_size_t()
        _check(ref().ref_ctx_key_shape(self.h, kind, rot, C.byref(parts), C.byref(kl)), "ref_ctx_key_shape")
        _check(ref().ref_ctx_key_words(self.h, kind, rot, C.byref(words)), "ref_ctx_key_words")
        out = np.zeros(parts.value * 2 * words.value, np.uint64)
        _check(ref().ref_ctx_key(self.h, kind, rot, out), "ref_ctx_key")
        return out, parts.value, kl.value

    def modraise(self, target_level, b, a):
        n = (target_level + 1) * self.N
        bo = np.zeros(n, np.uint64)
        ao = np.zeros(n, np.uint64)
        bo[: self.N] = np.asarray(b, dtype=np.uint64)[: self.N]
        ao[: self.N] = np.asarray(a, dtype=np.uint64)[: self.N]
        _check(ref().ref_modraise(self.h, target_level, bo, ao), "ref_modraise")
        return bo, ao

    def evalchebyshev(self, level, scale, coeffs, b, a, target_scale=0.0):
        """The reference's ckks_evalchebyshev_preconditioned: (b, a, out_level, out_scale)."""
        n = (level + 1) * self.N
        ob = np.zeros(n, np.uint64)
        oa = np.zeros(n, np.uint64)
        lvl, sc = C.c_size_t(), C.c_double()
        _check(ref().ref_evalchebyshev(self.h, level, float(scale), np.ascontiguousarray(coeffs, dtype=np.float64),
                                       len(coeffs), float(target_scale), np.ascontiguousarray(b[:n], dtype=np.uint64),
                                       np.ascontiguousarray(a[:n], dtype=np.uint64), C.byref(lvl), C.byref(sc), ob, oa),
               "ref_evalchebyshev")
        m = (lvl.value + 1) * self.N
        return ob[:m].copy(), oa[:m].copy(), lvl.value, sc.value

    def bts_info(self):
        """EvalMod bootstrap parameters of a bootstrapping context, with its EvalMod series."""
        v = [C.c_size_t() for _ in range(6)]
        sc, nc = C.c_double(), C.c_size_t()
        _check(ref().ref_bts_info(self.h, *[C.byref(x) for x in v], C.byref(sc), C.byref(nc)), "ref_bts_info")
        coeffs = np.zeros(nc.value, np.float64)
        _check(ref().ref_bts_evalmod_coeffs(self.h, coeffs), "ref_bts_evalmod_coeffs")
        keys = ("s2c_depth", "depth", "evalmod_log_scale", "double_angle", "active_slots", "slots")
        out = {k: x.value for k, x in zip(keys, v)}
        out["scale"] = sc.value
        out["coeffs"] = coeffs
        return out

    def bootstrap_evalmod(self, level, scale, b, a):
        """The reference's EvalMod bootstrap of one packed ciphertext: (out0, out1, level, scale)."""
        n = (self.N) * len(self.q)
        bufs = [np.zeros(n, np.uint64) for _ in range(4)]
        lvl, sc = C.c_size_t(), C.c_double()
        m = (level + 1) * self.N
        _check(ref().ref_bootstrap_evalmod(self.h, level, float(scale), np.ascontiguousarray(b[:m], dtype=np.uint64),
                                           np.ascontiguousarray(a[:m], dtype=np.uint64), *bufs, C.byref(lvl),
                                           C.byref(sc)), "ref_bootstrap_evalmod")
        k = (lvl.value + 1) * self.N
        return (bufs[0][:k].copy(), bufs[1][:k].copy()), (bufs[2][:k].copy(), bufs[3][:k].copy()), lvl.value, sc.value

    def secret_coeffs(self, sparse=False):
        """The context's ternary secret (or, when sparse, its bootstrapping sparse secret) as N
        int8 coefficients."""
        return _secret_from_ntt(self.h, self.N, len(self.q), low=sparse)

    def bootstrap_pair(self, level, scale0, scale1, ct0, ct1):
        """The reference's pair bootstrap (ckks_batch_bootstrap_evalmod_inplace) of ct0 = (b, a)
        and ct1: (out0, out1, level, scale)."""
        n = self.N * len(self.q)
        bufs = [np.zeros(n, np.uint64) for _ in range(4)]
        lvl, sc = C.c_size_t(), C.c_double()
        m = (level + 1) * self.N
        ins = [np.ascontiguousarray(x[:m], dtype=np.uint64) for x in (ct0[0], ct0[1], ct1[0], ct1[1])]
        _check(ref().ref_bootstrap_pair(self.h, level, float(scale0), float(scale1), *ins, *bufs, C.byref(lvl),
                                        C.byref(sc)), "ref_bootstrap_pair")
        k = (lvl.value + 1) * self.N
        return (bufs[0][:k].copy(), bufs[1][:k].copy()), (bufs[2][:k].copy(), bufs[3][:k].copy()), lvl.value, sc.value

    def bootstrap_pair_layer_seconds(self, level, scale, ct0, ct1, pairs, threads=0):
        """Wall time of `pairs` reference pair bootstraps on copies of ct0 = (b, a) and ct1, run as
        the reference's xboot_state_inplace runs the pairs of a state (OpenMP dynamic over pairs,
        src/ckks/operations/circuits/aes/ckks_aes_ctr.cpp:556-574) on `threads` threads (0: the
        OpenMP default).  The outputs are discarded."""
        R = ref()
        R.ref_bootstrap_pair_layer.argtypes = [C.c_void_p, C.c_size_t, C.c_double] + [u64p] * 4 + \
            [C.c_size_t, C.c_int, C.POINTER(C.c_double)]
        m = (level + 1) * self.N
        ins = [np.ascontiguousarray(x[:m], dtype=np.uint64) for x in (ct0[0], ct0[1], ct1[0], ct1[1])]
        sec = C.c_double()
        _check(R.ref_bootstrap_pair_layer(self.h, level, float(scale), *ins, pairs, threads, C.byref(sec)),
               "ref_bootstrap_pair_layer")
        return sec.value

    def xboot_key_bits(self, expanded_key, first_round_key_level=4):
        """The reference's encrypted expanded-key bits for the XBOOT AES
        (ckks_aes128_encrypt_expanded_round_key_bits): ([(b, a)] x 1408, scales, levels)."""
        s2c = self.bts_info()["s2c_depth"]
        top = s2c + first_round_key_level
        words = 2 * self.N * (128 * (top + 1) + 1280 * (s2c + 1))
        out = np.zeros(words, np.uint64)
        scales = np.zeros(1408, np.float64)
        levels = np.zeros(1408, np.uintp)
        _check(ref().ref_xboot_key_bits(self.h, bytes(expanded_key), first_round_key_level, out, scales, levels),
               "ref_xboot_key_bits")
        bits, off = [], 0
        for k in range(1408):
            m = (int(levels[k]) + 1) * self.N
            bits.append((out[off:off + m], out[off + m:off + 2 * m]))
            off += 2 * m
        return bits, scales, levels.astype(np.int64)

    def xboot_initial_state(self, keys, key_scales, key_level, counters, blocks):
        """The XBOOT initial state restated on the reference's operations
        (ref_xboot_initial_state): ([(b, a)] x 128, level, scales)."""
        n = (key_level + 1) * self.N
        flat = np.concatenate([np.concatenate([np.asarray(b[:n], np.uint64), np.asarray(a[:n], np.uint64)])
                               for b, a in keys])
        out = np.zeros(128 * 2 * n, np.uint64)
        lvl = C.c_size_t()
        sc = np.zeros(128, np.float64)
        R = ref()
        R.ref_xboot_initial_state.argtypes = [C.c_void_p, u64p, f64p, C.c_size_t, C.c_char_p, C.c_size_t, u64p,
                                              C.POINTER(C.c_size_t), f64p]
        _check(R.ref_xboot_initial_state(self.h, flat, np.ascontiguousarray(key_scales, np.float64), key_level,
                                         bytes(counters), blocks, out, C.byref(lvl), sc), "ref_xboot_initial_state")
        m = (lvl.value + 1) * self.N
        return [(out[2 * k * m:(2 * k + 1) * m].copy(), out[(2 * k + 1) * m:(2 * k + 2) * m].copy())
                for k in range(128)], lvl.value, sc

    def xboot_linear(self, state, in_scales, level, keys, key_level, mix):
        """ShiftRows, MixColumns (when mix) and AddRoundKey restated on the reference's operations
        (ref_xboot_linear): ([(b, a)] x 128, scales)."""
        n, kn = (level + 1) * self.N, (key_level + 1) * self.N
        flat = np.concatenate([np.concatenate([np.asarray(b[:n], np.uint64), np.asarray(a[:n], np.uint64)])
                               for b, a in state])
        kflat = np.concatenate([np.concatenate([np.asarray(b[:kn], np.uint64), np.asarray(a[:kn], np.uint64)])
                                for b, a in keys])
        out = np.zeros(128 * 2 * n, np.uint64)
        sc = np.zeros(128, np.float64)
        R = ref()
        R.ref_xboot_linear.argtypes = [C.c_void_p, u64p, f64p, C.c_size_t, u64p, C.c_size_t, C.c_int, u64p, f64p]
        _check(R.ref_xboot_linear(self.h, flat, np.ascontiguousarray(in_scales, np.float64), level, kflat, key_level,
                                  1 if mix else 0, out, sc), "ref_xboot_linear")
        return [(out[2 * k * n:(2 * k + 1) * n].copy(), out[(2 * k + 1) * n:(2 * k + 2) * n].copy())
                for k in range(128)], sc

    def build_scaled_s2c(self, ratio):
        """Build the SlotToCoeff plan for inputs at `ratio` x the parameter scale; its stages are
        then plan 100 + ratio for stages() / stage()."""
        _check(ref().ref_build_scaled_s2c(self.h, int(ratio)), "ref_build_scaled_s2c")
        return 100 + int(ratio)

    def aes_key_bits(self, expanded_key, active_blocks):
        """The reference's encrypted expanded-key bits: (flat [bit][b, a][limbs][N], scales, key level)."""
        kl = 2
        out = np.zeros(1408 * 2 * (kl + 1) * self.N, np.uint64)
        scales = np.zeros(1408, np.float64)
        lv = C.c_size_t()
        _check(ref().ref_aes_key_bits(self.h, bytes(expanded_key), active_blocks, out, scales, C.byref(lv)),
               "ref_aes_key_bits")
        assert lv.value == kl
        return out, scales, lv.value

    def aes_ctr(self, key_flat, key_scales, key_level, counters, ciphertexts, active_blocks):
        """The reference's AES-CTR on lazy bits: 128 x (b, a, level, scale)."""
        out = np.zeros(128 * 2 * len(self.q) * self.N, np.uint64)
        lv = np.zeros(128, np.uintp)
        sc = np.zeros(128, np.float64)
        _check(ref().ref_aes_ctr(self.h, key_flat, np.ascontiguousarray(key_scales, np.float64), key_level,
                                 bytes(counters), bytes(ciphertexts), active_blocks, out, lv, sc), "ref_aes_ctr")
        res, off = [], 0
        for k in range(128):
            m = (int(lv[k]) + 1) * self.N
            res.append((out[off:off + m].copy(), out[off + m:off + 2 * m].copy(), int(lv[k]), float(sc[k])))
            off += 2 * m
        return res

    def decrypt(self, level, scale, b, a):
        """The reference's ckks_decrypt: complex slot values."""
        re = np.zeros(self.N // 2)
        im = np.zeros(self.N // 2)
        n = (level + 1) * self.N
        _check(ref().ref_decrypt(self.h, level, float(scale), np.ascontiguousarray(b[:n], np.uint64),
                                 np.ascontiguousarray(a[:n], np.uint64), re, im), "ref_decrypt")
        return re + 1j * im

    def encode(self, re, im, scale, level):
        """The reference's ckks_encode, coefficient form, (level+1)*N residues."""
        out = np.zeros((level + 1) * self.N, np.uint64)
        _check(ref().ref_encode(self.h, np.ascontiguousarray(re, np.float64), np.ascontiguousarray(im, np.float64),
                                float(scale), level, out), "ref_encode")
        return out

    def walsh_sbox_layer_seconds(self, block_count, level, scale, bits, instances, threads=0):
        """Wall time of `instances` reference S-box calls on the 8 bit ciphertexts `bits`, run as
        the reference's SubBytes runs its byte positions (OpenMP over instances)."""
        n = (level + 1) * self.N
        flat = np.concatenate([np.concatenate([np.asarray(b[:n], np.uint64), np.asarray(a[:n], np.uint64)])
                               for b, a in bits])
        sec = C.c_double()
        _check(ref().ref_walsh_sbox_layer(self.h, block_count, level, float(scale), flat, instances, threads,
                                          C.byref(sec)), "ref_walsh_sbox_layer")
        return sec.value

    def walsh_sbox(self, block_count, level, scale, bits):
        """The reference's mask-packed Walsh S-box on 8 bit ciphertexts [(b, a)] x 8:
        returns [(b, a, level, scale)] x 8."""
        n = (level + 1) * self.N
        flat = np.concatenate([np.concatenate([np.asarray(b[:n], np.uint64), np.asarray(a[:n], np.uint64)])
                               for b, a in bits])
        out = np.zeros(16 * len(self.q) * self.N, np.uint64)
        lv = np.zeros(8, np.uintp)
        sc = np.zeros(8, np.float64)
        _check(ref().ref_walsh_sbox(self.h, block_count, level, float(scale), flat, out, lv, sc), "ref_walsh_sbox")
        res, off = [], 0
        for k in range(8):
            m = (int(lv[k]) + 1) * self.N
            res.append((out[off:off + m].copy(), out[off + m:off + 2 * m].copy(), int(lv[k]), float(sc[k])))
            off += 2 * m
        return res

    def dense_to_sparse(self, b, a):
        b = np.ascontiguousarray(b[: self.N], dtype=np.uint64).copy()
        a = np.ascontiguousarray(a[: self.N], dtype=np.uint64).copy()
        _check(ref().ref_dense_to_sparse(self.h, b, a), "ref_dense_to_sparse")
        return b, a

    def sparse_to_dense(self, level, b, a):
        n = (level + 1) * self.N
        b = np.ascontiguousarray(b[:n], dtype=np.uint64).copy()
        a = np.ascontiguousarray(a[:n], dtype=np.uint64).copy()
        _check(ref().ref_sparse_to_dense(self.h, level, b, a), "ref_sparse_to_dense")
        return b, a
