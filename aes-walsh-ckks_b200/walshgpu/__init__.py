"""Python binding of libwalshgpu.so (include/walsh_gpu.h) over ctypes.

The library is the product: every operation here is one C-ABI call that launches sm_100a
kernels.  There is no CPU fallback -- importing this module fails loudly when the library is
missing, and every call raises when the library reports an error.

Device buffers are torch tensors (dtype int64 holding the uint64 residues bit for bit);
torch only provides memory and the current CUDA stream.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "libwalshgpu.so")

WG_KEY_RELIN = 0
WG_KEY_CONJ = 1
WG_KEY_ROTATION = 2
WG_KEY_DENSE_TO_SPARSE = 3
WG_KEY_SPARSE_TO_DENSE = 4


class WalshGpuError(RuntimeError):
    """Raised for a non-zero status of the C ABI; `code` is the WG_ERR_* value."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class InvalidArgument(WalshGpuError, ValueError):
    """WG_ERR_INVALID -- the reference raises std::invalid_argument here."""


def build(force: bool = False) -> str:
    """Compile libwalshgpu.so in-tree for sm_100a (nvcc cross-compiles without a GPU)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-j8", "-C", PKG], check=True)
    return LIB_PATH


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libwalshgpu.so is not built ({LIB_PATH}); run walshgpu.build()")
        L = C.CDLL(LIB_PATH)
        vp, sz, u64 = C.c_void_p, C.c_size_t, C.c_uint64
        L.wg_last_error.restype = C.c_char_p
        L.wg_version.restype = C.c_int
        L.wg_encode_slots.argtypes = [u64, vp, vp, C.c_double, vp, sz, vp]
        L.wg_find_primes.argtypes = [vp, sz, vp, sz, u64, vp, vp]
        L.wg_ctx_create.argtypes = [u64, vp, sz, vp, sz, sz, C.c_int, C.POINTER(vp)]
        L.wg_ctx_destroy.argtypes = [vp]
        L.wg_ctx_destroy.restype = None
        L.wg_ctx_set_key.argtypes = [vp, C.c_int, C.c_int64, vp, sz, sz]
        L.wg_ctx_has_key.argtypes = [vp, C.c_int, C.c_int64]
        L.wg_ctx_reserve.argtypes = [vp, vp]
        L.wg_ctx_trim.argtypes = [vp, vp]
        L.wg_ctx_workspace_words.argtypes = [vp]
        L.wg_ctx_workspace_words.restype = sz
        for f in (L.wg_ntt_forward, L.wg_ntt_inverse):
            f.argtypes = [vp, vp, sz, sz, C.c_int, sz, sz, vp]
        L.wg_ntt_tuning.argtypes = [vp, vp, vp, vp]
        L.wg_ct_wire_bytes.argtypes = [u64, sz, sz]
        L.wg_ct_wire_bytes.restype = sz
        L.wg_ct_wire_encode.argtypes = [u64, vp, sz, sz, vp, C.c_double, C.c_int, C.c_int, vp, sz]
        L.wg_ct_wire_decode.argtypes = [vp, sz, u64, vp, sz, vp, sz, vp, vp, vp, vp, vp]
        L.wg_serve_budget_create.argtypes = [sz, vp]
        L.wg_serve_budget_destroy.argtypes = [vp]
        L.wg_serve_budget_destroy.restype = None
        L.wg_evalmod_fit.argtypes = [C.c_double, sz, sz, C.c_double, sz, C.c_double, vp, vp, vp, vp]
        L.wg_evalmod_k_bound.argtypes = [sz, sz, C.c_double, vp]
        L.wg_dft_plan_describe.argtypes = [u64, vp, sz, vp, sz] + [vp] * 8
        L.wg_dft_plan_create.argtypes = [vp, vp, vp, sz, vp, vp]
        L.wg_lt_stage_info.argtypes = [vp] * 7
        L.wg_lt_stage_download.argtypes = [vp, vp, vp, vp]
        L.wg_ntt_set_geometry.argtypes = [vp, C.c_int, C.c_int, C.c_int]
        L.wg_set_ntt_fusion.argtypes = [vp, C.c_int]
        L.wg_keyswitch.argtypes = [vp, sz, vp, C.c_int, C.c_int64, vp, vp, C.c_int, C.c_int, vp]
        L.wg_rotate.argtypes = [vp, sz, vp, vp, C.c_int64, vp]
        L.wg_rotate_noalloc.argtypes = [vp, sz, vp, vp, C.c_int64, vp]
        L.wg_conjugate.argtypes = [vp, sz, vp, vp, vp]
        L.wg_rotate_many.argtypes = [vp, sz, vp, vp, vp, sz, vp, vp]
        L.wg_mul.argtypes = [vp, sz, vp, vp, vp, vp, vp, vp]
        L.wg_relin.argtypes = [vp, sz, vp, vp, vp, vp]
        L.wg_rescale.argtypes = [vp, sz, vp, sz, sz, vp]
        L.wg_add.argtypes = [vp, sz, vp, vp, sz, sz, vp]
        L.wg_sub.argtypes = [vp, sz, vp, vp, sz, sz, vp]
        L.wg_batch_mul_relin_rescale_rotate.argtypes = [vp, sz, vp, vp, vp, vp, vp, vp, vp]
        L.wg_sequence_mul_relin_rescale_rotate.argtypes = [vp, sz, vp, vp, vp, vp, vp, vp, vp]
        L.wg_modraise.argtypes = [vp, sz, sz, vp, vp, vp]
        L.wg_dense_to_sparse.argtypes = [vp, sz, vp, vp, vp]
        L.wg_sparse_to_dense.argtypes = [vp, sz, vp, vp, vp, vp]
        L.wg_evalchebyshev.argtypes = [vp, sz, sz, C.c_double, vp, sz, C.c_double, C.c_double, vp, vp, vp, vp,
                                       C.POINTER(C.c_size_t), C.POINTER(C.c_double), vp]
        L.wg_bootstrap_evalmod.argtypes = [vp, vp, vp, sz, vp, sz, vp, sz, sz, vp, vp, vp, vp, vp, vp,
                                           C.POINTER(C.c_size_t), C.POINTER(C.c_double), vp]
        L.wg_walsh_sbox.argtypes = [vp, vp, vp, sz, vp, sz, vp, sz, sz, sz, sz, C.c_double, vp, vp, vp, vp, vp, vp, vp]
        for f in (L.wg_aes_ctr_walsh, L.wg_aes_ctr_walsh_plain):
            f.argtypes = [vp, vp, vp, sz, vp, sz, vp, sz, vp, sz, sz, sz, vp, vp, vp, sz, C.c_char_p, C.c_char_p, sz,
                          vp, vp, vp, vp, vp]
        L.wg_batch_plan_create.argtypes = [vp, sz, vp, vp, vp, vp, vp, vp, C.POINTER(vp)]
        L.wg_xboot_sbox.argtypes = [vp, sz, sz, C.c_double, vp, vp, vp, vp, vp, vp, vp]
        L.wg_xboot_sbox_coefficients.argtypes = [vp]
        L.wg_bootstrap_pair.argtypes = [vp, vp, vp, sz, vp, sz, vp, sz, sz, C.c_double, vp, vp, vp, vp,
                                        C.POINTER(C.c_size_t), C.POINTER(C.c_double), vp]
        L.wg_aes_ctr_xboot.argtypes = [vp, vp, vp, sz, vp, sz, vp, sz, vp, vp, vp, vp, C.c_char_p, C.c_char_p, sz,
                                       vp, vp, vp, vp, vp]
        L.wg_serve_create.argtypes = [vp, vp, vp, sz, vp, sz, vp, sz, vp, sz, sz, sz, vp, vp, vp, sz, vp,
                                      C.POINTER(vp)]
        L.wg_xboot_initial_state.argtypes = [vp, vp, vp, vp, vp, vp, C.c_char_p, sz, vp, vp, C.POINTER(C.c_size_t),
                                             vp, vp]
        L.wg_xboot_linear_layer.argtypes = [vp, sz, vp, vp, vp, vp, vp, vp, C.c_int, vp, vp, vp, vp]
        L.wg_keygen_switch_key.argtypes = [vp, C.c_int, C.c_int64, vp, vp, vp, C.c_uint64, C.c_double, vp, vp]
        L.wg_keygen_secret_switch.argtypes = [vp, C.c_int, vp, vp, vp, vp, C.c_uint64, C.c_double, vp, vp]
        L.wg_bundle_save.argtypes = [vp, C.c_char_p, vp, sz]
        L.wg_bundle_load.argtypes = [vp, C.c_char_p, vp, sz, C.POINTER(C.c_size_t)]
        L.wg_decrypt_decode.argtypes = [vp, sz, sz, vp, vp, vp, vp, vp, vp, vp, vp]
        L.wg_encode_slots_device.argtypes = [vp, sz, sz, C.c_double, vp, vp, vp, C.c_int, vp]
        L.wg_encrypt_symmetric.argtypes = [vp, sz, sz, vp, vp, vp, vp, C.c_uint64, C.c_double, vp, vp, vp]
        L.wg_aes_walsh_encrypt_round_key_bits.argtypes = [vp, vp, vp, sz, vp, C.c_uint64, C.c_double, vp, vp, vp,
                                                          vp, vp]
        L.wg_aes_xboot_encrypt_round_key_bits.argtypes = [vp, vp, vp, sz, vp, C.c_uint64, C.c_double, vp, vp, vp,
                                                          vp, vp]
        L.wg_serve_create_xboot.argtypes = [vp, vp, vp, sz, vp, sz, vp, sz, vp, vp, vp, vp, vp, C.POINTER(vp)]
        L.wg_serve_submit.argtypes = [vp, C.c_char_p, C.c_char_p, sz, vp, vp, C.POINTER(C.c_uint64)]
        L.wg_serve_wait.argtypes = [vp, C.c_uint64, C.c_double, vp]
        L.wg_serve_destroy.argtypes = [vp]
        L.wg_serve_destroy.restype = None
        L.wg_batch_plan_launch.argtypes = [vp, vp]
        L.wg_batch_plan_destroy.argtypes = [vp]
        L.wg_batch_plan_destroy.restype = None
        L.wg_lt_stage_create.argtypes = [vp, sz, sz, vp, vp, sz, sz, C.c_int, C.POINTER(vp)]
        L.wg_lt_stage_destroy.argtypes = [vp]
        L.wg_lt_stage_destroy.restype = None
        L.wg_lt_stage_apply.argtypes = [vp, vp, sz, vp, vp, vp]
        L.wg_launch_count.argtypes = [C.c_int]
        L.wg_launch_count.restype = C.c_uint64
        L.wg_probe_begin.argtypes = [C.c_int, C.c_int]
        L.wg_probe_end.argtypes = [C.POINTER(C.c_uint64), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.wg_host_stats.argtypes = [C.POINTER(C.c_uint64), C.c_size_t]
        L.wg_malloc.argtypes = [C.POINTER(vp), sz]
        L.wg_free.argtypes = [vp]
        L.wg_memcpy_htod.argtypes = [vp, vp, sz, vp]
        L.wg_memcpy_dtoh.argtypes = [vp, vp, sz, vp]
        L.wg_stream_synchronize.argtypes = [vp]
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != 0:
        msg = lib().wg_last_error().decode()
        if rc == -1:
            raise InvalidArgument(rc, msg)
        raise WalshGpuError(rc, msg)


def _ptr(t) -> int:
    """Device pointer of a torch tensor (or an int already holding one)."""
    if t is None:
        return 0
    if isinstance(t, int):
        return t
    return t.data_ptr()


def _stream(stream=None) -> int:
    if stream is not None:
        return stream if isinstance(stream, int) else stream.cuda_stream
    import torch

    return torch.cuda.current_stream().cuda_stream


def _u64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint64))


KCLASS = {"ntt": 0, "modup": 1, "keymac": 2, "moddown": 3, "combine": 4, "elementwise": 5, "walsh": 6,
          "giant": 7}


def launch_count(kernel_class=-1) -> int:
    """Kernel launches the library issued so far (all classes by default)."""
    return int(lib().wg_launch_count(kernel_class))


def probe_begin(kernel_class, max_launches=60000):
    """Start CUDA-event timing of every launch of one kernel class."""
    _check(lib().wg_probe_begin(kernel_class, max_launches))


def xboot_sbox_coefficients():
    """[8][256] integer coefficients of the S-box output bits over the input-bit monomials."""
    out = np.zeros(8 * 256, np.int64)
    _check(lib().wg_xboot_sbox_coefficients(out.ctypes.data))
    return out.reshape(8, 256)


def host_stats() -> dict:
    """Host-side counters: slot encodings and their time, staged uploads, bytes, waits."""
    out = (C.c_uint64 * 5)()
    _check(lib().wg_host_stats(out, 5))
    return {"encodes": out[0], "encode_ms": out[1] / 1e6, "stages": out[2], "stage_bytes": out[3],
            "stage_wait_ms": out[4] / 1e6}


def probe_end():
    """Stop timing; returns (launches, total_ms, total_algorithmic_bytes)."""
    n, ms, by = C.c_uint64(), C.c_double(), C.c_double()
    _check(lib().wg_probe_end(C.byref(n), C.byref(ms), C.byref(by)))
    return n.value, ms.value, by.value


def memcpy_htod(dst, src_ptr, nbytes, stream=None):
    _check(lib().wg_memcpy_htod(_ptr(dst), src_ptr, nbytes, _stream(stream)))


def memcpy_dtoh(dst_ptr, src, nbytes, stream=None):
    _check(lib().wg_memcpy_dtoh(dst_ptr, _ptr(src), nbytes, _stream(stream)))


def find_primes(p_bits, q_bits, N):
    """Reference prime chain (find_p_and_q_primes): returns (p, q) as uint64 arrays."""
    pb, qb = _u64(p_bits), _u64(q_bits)
    p = np.zeros(len(pb), np.uint64)
    q = np.zeros(len(qb), np.uint64)
    _check(lib().wg_find_primes(pb.ctypes.data, len(pb), qb.ctypes.data, len(qb), int(N), p.ctypes.data,
                                q.ctypes.data))
    return p, q


def evalmod_fit(K, degree, double_angle, interval_radius, validation_points, prune_threshold):
    """The EvalMod Chebyshev series (host, 256-bit): {"coeffs", "max_error", "interval"}."""
    out = np.zeros(int(degree) + 1, np.float64)
    n = C.c_size_t()
    err = C.c_double()
    iv = np.zeros(2, np.float64)
    _check(lib().wg_evalmod_fit(float(K), int(degree), int(double_angle), float(interval_radius),
                                int(validation_points), float(prune_threshold), out.ctypes.data, C.byref(n),
                                C.byref(err), iv.ctypes.data))
    return {"coeffs": out[: n.value].copy(), "max_error": err.value, "interval": (iv[0], iv[1])}


def evalmod_k_bound(coefficients, hamming_weight, log2_failure):
    k = C.c_size_t()
    _check(lib().wg_evalmod_k_bound(int(coefficients), int(hamming_weight), float(log2_failure), C.byref(k)))
    return k.value


def ct_wire_encode(N, q, level, polys, scale, secret_owner=0, encoding_state=0) -> bytes:
    """The wire record of a ciphertext: polys = host residues [npolys][level + 1][N]."""
    qa = _u64(q)
    pa = _u64(polys)
    npolys = pa.size // ((level + 1) * int(N))
    n = lib().wg_ct_wire_bytes(int(N), int(level), npolys)
    out = np.zeros(n, np.uint8)
    _check(lib().wg_ct_wire_encode(int(N), qa.ctypes.data, int(level), npolys, pa.ctypes.data, float(scale),
                                   int(secret_owner), int(encoding_state), out.ctypes.data, n))
    return out.tobytes()


def ct_wire_decode(record, N, q):
    """(residues [npolys][level + 1][N] as a flat array, level, scale, secret_owner, encoding_state)
    of a wire record checked against the context's ring degree and Q moduli."""
    buf = np.frombuffer(bytes(record), dtype=np.uint8).copy()
    qa = _u64(q)
    out = np.zeros(3 * len(qa) * int(N), np.uint64)
    lv, npl, sc, ow, st = C.c_size_t(), C.c_size_t(), C.c_double(), C.c_int(), C.c_int()
    _check(lib().wg_ct_wire_decode(buf.ctypes.data, buf.size, int(N), qa.ctypes.data, len(qa), out.ctypes.data,
                                   out.size, C.byref(lv), C.byref(npl), C.byref(sc), C.byref(ow), C.byref(st)))
    return out[: npl.value * (lv.value + 1) * int(N)], lv.value, sc.value, ow.value, st.value


def to_device(arr, device="cuda"):
    """uint64 numpy array -> int64 torch tensor on the GPU (bit-identical)."""
    import torch

    return torch.from_numpy(_u64(arr).view(np.int64).copy()).to(device)


def encode_slots(N, re, im, scale, moduli) -> np.ndarray:
    """Host CKKS encoding of N/2 complex slots at `scale`: coefficient-form residues per modulus."""
    r = np.ascontiguousarray(re, dtype=np.float64)
    i = np.ascontiguousarray(im, dtype=np.float64)
    m = _u64(moduli)
    out = np.zeros(len(m) * int(N), np.uint64)
    _check(lib().wg_encode_slots(int(N), r.ctypes.data, i.ctypes.data, float(scale), m.ctypes.data, len(m),
                                 out.ctypes.data))
    return out


def to_host(t) -> np.ndarray:
    """int64 torch tensor -> uint64 numpy array (bit-identical)."""
    return t.detach().cpu().numpy().view(np.uint64).copy()


class LtStage:
    """One baby-step / giant-step linear-transform stage (diagonals device-resident)."""

    def __init__(self, ctx, level, indices, diagonals, baby_step_count, slot_count=0, rescale=False):
        self.ctx = ctx
        idx = _u64(indices)
        d = _u64(diagonals)
        h = C.c_void_p()
        _check(lib().wg_lt_stage_create(ctx.h, level, len(idx), idx.ctypes.data, d.ctypes.data, baby_step_count,
                                        slot_count, int(rescale), C.byref(h)))
        self.h = h
        self.level = level
        self.rescale = rescale

    def info(self):
        """{"level", "nterms", "baby", "slots", "rescale", "plaintext_scale"} of the stage."""
        lv, nt, bb, sl = C.c_size_t(), C.c_size_t(), C.c_size_t(), C.c_size_t()
        rs, ps = C.c_int(), C.c_double()
        _check(lib().wg_lt_stage_info(self.h, C.byref(lv), C.byref(nt), C.byref(bb), C.byref(sl), C.byref(rs),
                                      C.byref(ps)))
        return dict(level=lv.value, nterms=nt.value, baby=bb.value, slots=sl.value, rescale=bool(rs.value),
                    plaintext_scale=ps.value)

    def download(self):
        """(indices, diagonals [term][QP limbs][N]) in host memory."""
        inf = self.info()
        idx = np.zeros(inf["nterms"], np.uint64)
        d = np.zeros(inf["nterms"] * (inf["level"] + 1 + len(self.ctx.p)) * self.ctx.N, np.uint64)
        _check(lib().wg_lt_stage_download(self.ctx.h, self.h, idx.ctypes.data, d.ctypes.data))
        return idx, d

    @classmethod
    def from_handle(cls, ctx, h, level=None, rescale=None):
        """Wrap a stage handle the library created (wg_bundle_load)."""
        self = cls.__new__(cls)
        self.ctx, self.h, self.level, self.rescale = ctx, h, level, rescale
        return self

    def apply(self, bs, as_, stream=None):
        """Apply to a batch of ciphertexts (lists of device tensors), in place."""
        pb = np.ascontiguousarray([_ptr(t) for t in bs], dtype=np.uint64)
        pa = np.ascontiguousarray([_ptr(t) for t in as_], dtype=np.uint64)
        _check(lib().wg_lt_stage_apply(self.ctx.h, self.h, len(pb), pb.ctypes.data, pa.ctypes.data, _stream(stream)))

    def close(self):
        if getattr(self, "h", None):
            lib().wg_lt_stage_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DftLiteral(C.Structure):
    """wg_dft_literal: one homomorphic DFT to factorize into BSGS stages."""
    _fields_ = [("coeffs_to_slots", C.c_int), ("level", C.c_size_t), ("baby_step_count", C.c_size_t),
                ("log_bsgs_ratio", C.c_int), ("stage_count", C.c_size_t), ("group_sizes", C.c_void_p),
                ("group_bits", C.c_void_p), ("ngroups", C.c_size_t), ("merge_depths", C.c_void_p),
                ("nmerge", C.c_size_t), ("active_slots", C.c_size_t), ("transform_scale", C.c_double),
                ("input_selector_start", C.c_size_t), ("input_selector_size", C.c_size_t)]

    @classmethod
    def make(cls, coeffs_to_slots, level, transform_scale, scale_groups=(), stage_count=0, merge_depths=(),
             active_slots=0, baby_step_count=0, log_bsgs_ratio=1, input_selector=(0, 0)):
        lit = cls()
        lit._keep = [np.ascontiguousarray([len(g) for g in scale_groups], dtype=np.uintp),
                     np.ascontiguousarray([b for g in scale_groups for b in g], dtype=np.uintp),
                     np.ascontiguousarray(list(merge_depths), dtype=np.uintp)]
        lit.coeffs_to_slots = int(bool(coeffs_to_slots))
        lit.level = int(level)
        lit.baby_step_count = int(baby_step_count)
        lit.log_bsgs_ratio = int(log_bsgs_ratio)
        lit.stage_count = int(stage_count)
        lit.group_sizes = lit._keep[0].ctypes.data if len(scale_groups) else None
        lit.group_bits = lit._keep[1].ctypes.data if len(scale_groups) else None
        lit.ngroups = len(scale_groups)
        lit.merge_depths = lit._keep[2].ctypes.data if len(merge_depths) else None
        lit.nmerge = len(merge_depths)
        lit.active_slots = int(active_slots)
        lit.transform_scale = float(transform_scale)
        lit.input_selector_start, lit.input_selector_size = (int(input_selector[0]), int(input_selector[1]))
        return lit


def dft_plan_describe(N, q, literal, stage, diagonals=False):
    """One stage of the factorized DFT generated on the host (no device): its shape, indices
    and optionally its diagonals before encoding (complex [nterms][active slots])."""
    qa = _u64(q)
    ns, lv, nt, bb = C.c_size_t(), C.c_size_t(), C.c_size_t(), C.c_size_t()
    rs, ps = C.c_int(), C.c_double()
    _check(lib().wg_dft_plan_describe(int(N), qa.ctypes.data, len(qa), C.byref(literal), int(stage), C.byref(ns),
                                      C.byref(lv), C.byref(nt), C.byref(bb), C.byref(rs), C.byref(ps), None, None))
    idx = np.zeros(nt.value, np.uint64)
    slots = literal.active_slots or int(N) // 2
    d = np.zeros(2 * nt.value * slots, np.float64) if diagonals else None
    _check(lib().wg_dft_plan_describe(int(N), qa.ctypes.data, len(qa), C.byref(literal), int(stage), None, None,
                                      None, None, None, None, idx.ctypes.data, None if d is None else d.ctypes.data))
    out = dict(stages=ns.value, level=lv.value, nterms=nt.value, baby=bb.value, rescale=bool(rs.value),
               plaintext_scale=ps.value, indices=idx)
    if d is not None:
        out["diagonals"] = (d[0::2] + 1j * d[1::2]).reshape(nt.value, slots)
    return out


class BootstrapParams(C.Structure):
    """wg_bootstrap_params."""
    _fields_ = [("s2c_depth", C.c_size_t), ("depth", C.c_size_t), ("evalmod_log_scale", C.c_size_t),
                ("double_angle", C.c_size_t), ("active_slots", C.c_size_t), ("slots", C.c_size_t),
                ("scale", C.c_double)]


class ServeConfig(C.Structure):
    """wg_serve_config."""
    _fields_ = [("workers", C.c_size_t), ("hbm_budget_bytes", C.c_size_t), ("eval_bytes", C.c_size_t),
                ("max_blocks", C.c_size_t), ("batch_window_ms", C.c_double), ("priority", C.c_int),
                ("budget", C.c_void_p)]


class ServeBudget:
    """A device-memory budget shared by several servers (wg_serve_budget_create); keep it alive
    until the servers using it are closed."""

    def __init__(self, nbytes):
        h = C.c_void_p()
        _check(lib().wg_serve_budget_create(int(nbytes), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().wg_serve_budget_destroy(self.h)
            self.h = None


class ServeResult(C.Structure):
    """wg_serve_result."""
    _fields_ = [("status", C.c_int), ("block_offset", C.c_size_t), ("active_blocks", C.c_size_t),
                ("batch_requests", C.c_size_t), ("batch_blocks", C.c_size_t), ("queue_ms", C.c_double),
                ("latency_ms", C.c_double), ("out_level", C.c_size_t * 128), ("out_scale", C.c_double * 128)]


WG_NOT_READY = 1


class Server:
    """Continuous-batching AES-CTR service (wg_serve_*): requests of counter blocks (an even
    number for Walsh evaluations) are packed in arrival order into shared evaluations that
    `workers` streams run concurrently; Server.xboot(...) serves XBOOT evaluations.  The stages,
    key bits and coefficients must outlive the server."""

    def __init__(self, ctx, params, s2c, s2c_x2, c2s, coeffs, packing_block_count, packed_segment_count, key_bits,
                 key_scales, key_level, workers=2, hbm_budget_bytes=0, eval_bytes=0, max_blocks=0,
                 batch_window_ms=0.0, priority=0, budget=None):
        arr = lambda ts: np.ascontiguousarray([_ptr(t) for t in ts], dtype=np.uint64)
        hs = lambda sts: np.ascontiguousarray([st.h.value for st in sts], dtype=np.uint64)
        # kept alive with the server: the library holds their addresses
        self._keep = (params, s2c, s2c_x2, c2s, key_bits)
        self._kb, self._ka = arr([x[0] for x in key_bits]), arr([x[1] for x in key_bits])
        self._ps, self._ps2, self._pc = hs(s2c), hs(s2c_x2), hs(c2s)
        self._cf = np.ascontiguousarray(coeffs, dtype=np.float64)
        self._ks = np.ascontiguousarray(key_scales, dtype=np.float64)
        cfg = ServeConfig(workers, hbm_budget_bytes, eval_bytes, max_blocks, batch_window_ms, int(priority),
                          None if budget is None else budget.h.value)
        h = C.c_void_p()
        _check(lib().wg_serve_create(ctx.h, C.byref(params), self._ps.ctypes.data, len(self._ps), self._ps2.ctypes.data,
                                     len(self._ps2), self._pc.ctypes.data, len(self._pc), self._cf.ctypes.data,
                                     len(self._cf), packing_block_count, packed_segment_count, self._kb.ctypes.data,
                                     self._ka.ctypes.data, self._ks.ctypes.data, key_level, C.byref(cfg), C.byref(h)))
        self.h = h
        self._outs = {}

    @classmethod
    def xboot(cls, ctx, params, s2c, c2s, coeffs, key_bits, key_scales, key_levels, workers=2, hbm_budget_bytes=0,
              eval_bytes=0, max_blocks=0, batch_window_ms=0.0, priority=0, budget=None):
        """The service over XBOOT evaluations (wg_serve_create_xboot): requests of 1..active-slot
        blocks, block b of an evaluation in slot b."""
        self = cls.__new__(cls)
        arr = lambda ts: np.ascontiguousarray([_ptr(t) for t in ts], dtype=np.uint64)
        hs = lambda sts: np.ascontiguousarray([st.h.value for st in sts], dtype=np.uint64)
        self._keep = (params, s2c, c2s, key_bits)
        self._kb, self._ka = arr([x[0] for x in key_bits]), arr([x[1] for x in key_bits])
        self._ps, self._pc = hs(s2c), hs(c2s)
        self._cf = np.ascontiguousarray(coeffs, dtype=np.float64)
        self._ks = np.ascontiguousarray(key_scales, dtype=np.float64)
        self._kl = np.ascontiguousarray(key_levels, dtype=np.uintp)
        cfg = ServeConfig(workers, hbm_budget_bytes, eval_bytes, max_blocks, batch_window_ms, int(priority),
                          None if budget is None else budget.h.value)
        h = C.c_void_p()
        _check(lib().wg_serve_create_xboot(ctx.h, C.byref(params), self._ps.ctypes.data, len(self._ps),
                                           self._pc.ctypes.data, len(self._pc), self._cf.ctypes.data, len(self._cf),
                                           self._kb.ctypes.data, self._ka.ctypes.data, self._ks.ctypes.data,
                                           self._kl.ctypes.data, C.byref(cfg), C.byref(h)))
        self.h = h
        self._outs = {}
        return self

    def submit(self, counters, ciphertexts, out_bits):
        """Queue a request (bytes of `blocks` counter and ciphertext blocks, 128 (b, a) device
        tensors for its output bits); returns its id."""
        blocks = len(counters) // 16
        ob = np.ascontiguousarray([_ptr(x[0]) for x in out_bits], dtype=np.uint64)
        oa = np.ascontiguousarray([_ptr(x[1]) for x in out_bits], dtype=np.uint64)
        rid = C.c_uint64()
        _check(lib().wg_serve_submit(self.h, bytes(counters), bytes(ciphertexts), blocks, ob.ctypes.data,
                                     oa.ctypes.data, C.byref(rid)))
        self._outs[rid.value] = out_bits
        return rid.value

    def wait(self, rid, timeout=-1.0):
        """The finished request's result (dict), or None on timeout."""
        r = ServeResult()
        rc = lib().wg_serve_wait(self.h, rid, float(timeout), C.byref(r))
        if rc == WG_NOT_READY:
            return None
        _check(rc)
        self._outs.pop(rid, None)
        if r.status != 0:
            raise WalshGpuError(r.status, lib().wg_last_error().decode())
        return {"block_offset": r.block_offset, "active_blocks": r.active_blocks,
                "batch_requests": r.batch_requests, "batch_blocks": r.batch_blocks, "queue_ms": r.queue_ms,
                "latency_ms": r.latency_ms, "levels": list(r.out_level), "scales": list(r.out_scale)}

    def close(self):
        if getattr(self, "h", None):
            lib().wg_serve_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchPlan:
    """The batched mul + relin + rescale + rotate pipeline planned once for fixed device buffers
    and captured as a CUDA graph (wg_batch_plan_*); launch() replays it on a stream."""

    def __init__(self, ctx, levels, xb, xa, yb, ya, rots):
        self.ctx = ctx
        lv = np.ascontiguousarray(levels, dtype=np.uintp)
        arr = lambda ts: np.ascontiguousarray([_ptr(t) for t in ts], dtype=np.uint64)
        pxb, pxa, pyb, pya = arr(xb), arr(xa), arr(yb), arr(ya)
        r = np.ascontiguousarray(rots, dtype=np.int64)
        h = C.c_void_p()
        _check(lib().wg_batch_plan_create(ctx.h, len(lv), lv.ctypes.data, pxb.ctypes.data, pxa.ctypes.data,
                                          pyb.ctypes.data, pya.ctypes.data, r.ctypes.data, C.byref(h)))
        self.h = h
        self._keep = (xb, xa, yb, ya)  # the graph reads and writes these buffers

    def launch(self, stream=None):
        _check(lib().wg_batch_plan_launch(self.h, _stream(stream)))

    def close(self):
        if getattr(self, "h", None):
            lib().wg_batch_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """Device-resident CKKS context (moduli, twiddles, base-change tables, keys)."""

    def __init__(self, N, q, p, dnum, device: int = 0):
        self.N = int(N)
        self.q = _u64(q)
        self.p = _u64(p)
        self.dnum = int(dnum)
        self.device = device
        self.alpha = (len(self.q) + self.dnum - 1) // self.dnum
        h = C.c_void_p()
        _check(lib().wg_ctx_create(self.N, self.q.ctypes.data, len(self.q), self.p.ctypes.data, len(self.p),
                                   self.dnum, device, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().wg_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nq(self):
        return len(self.q)

    @property
    def np_(self):
        return len(self.p)

    def parts(self, level):
        return min(self.dnum, (level + self.alpha) // self.alpha)

    def set_key(self, kind, key, rotation=0, parts=None, key_level=None):
        if kind == WG_KEY_DENSE_TO_SPARSE:  # compact q0/p0 key: one level-0 part
            key_level, parts = 0, 1
        kl = self.nq - 1 if key_level is None else key_level
        parts = self.parts(kl) if parts is None else parts
        k = _u64(key)
        expect = 4 * self.N if kind == WG_KEY_DENSE_TO_SPARSE else parts * 2 * (kl + 1 + self.np_) * self.N
        if k.size != expect:
            raise ValueError(f"key has {k.size} words, expected {expect}")
        _check(lib().wg_ctx_set_key(self.h, kind, int(rotation), k.ctypes.data, parts, kl))

    def has_key(self, kind, rotation=0):
        return bool(lib().wg_ctx_has_key(self.h, kind, int(rotation)))

    def reserve(self, stream=None):
        _check(lib().wg_ctx_reserve(self.h, _stream(stream)))

    def workspace_words(self):
        """Scratch words one in-flight single operation uses on a stream."""
        return int(lib().wg_ctx_workspace_words(self.h))

    def trim(self, stream=None):
        """Free the stream's scratch and the cached scratch chunks (after the stream's work)."""
        _check(lib().wg_ctx_trim(self.h, _stream(stream)))

    # --- operations on device buffers -------------------------------------------------
    def ntt_forward(self, poly, limbs, first=0, basis=0, polys=1, stride=0, stream=None):
        _check(lib().wg_ntt_forward(self.h, _ptr(poly), limbs, first, basis, polys, stride, _stream(stream)))

    def ntt_inverse(self, poly, limbs, first=0, basis=0, polys=1, stride=0, stream=None):
        _check(lib().wg_ntt_inverse(self.h, _ptr(poly), limbs, first, basis, polys, stride, _stream(stream)))

    def dft_plan(self, literal, stream=None):
        """Generate the factorized DFT's stages on this context's device: a list of LtStage."""
        hs = (C.c_void_p * 64)()
        n = C.c_size_t()
        _check(lib().wg_dft_plan_create(self.h, C.byref(literal), hs, 64, C.byref(n), _stream(stream)))
        out = []
        for i in range(n.value):
            st = LtStage.from_handle(self, C.c_void_p(hs[i]))
            inf = st.info()
            st.level, st.rescale = inf["level"], inf["rescale"]
            out.append(st)
        return out

    NTT_GEOMETRIES = ("8 residues/thread, staged twiddles", "8 residues/thread, table twiddles",
                      "16 residues/thread, staged twiddles", "16 residues/thread, table twiddles")

    def ntt_tuning(self):
        """The NTT autotuner's result: {"chosen": [[fwd rows, fwd cols], [inv rows, inv cols]],
        "ms": array [direction][phase][geometry], "limbs": limbs of the timed batch}."""
        chosen = np.zeros(4, np.int32)
        ms = np.zeros(16, np.float32)
        limbs = C.c_int()
        _check(lib().wg_ntt_tuning(self.h, chosen.ctypes.data, ms.ctypes.data, C.byref(limbs)))
        return {"chosen": chosen.reshape(2, 2).tolist(), "ms": ms.reshape(2, 2, 4), "limbs": limbs.value}

    def set_ntt_geometry(self, direction, phase, geometry):
        """Pin the NTT geometry of (direction 0 fwd / 1 inv, phase 0 rows / 1 cols); -1 restores
        the tuned choice."""
        _check(lib().wg_ntt_set_geometry(self.h, int(direction), int(phase), int(geometry)))

    def set_ntt_fusion(self, mode):
        """Key switches and rescales with their base changes fused into the NTT column phases
        and their last element-wise steps into the row-phase epilogue: 0 never, 1 when the
        launch fills the device (default; True maps here), 2 always; the words are the same."""
        _check(lib().wg_set_ntt_fusion(self.h, int(mode)))

    def keyswitch(self, level, key_term, kind, b, a, b_add=True, a_add=False, rotation=0, stream=None):
        _check(lib().wg_keyswitch(self.h, level, _ptr(key_term), kind, int(rotation), _ptr(b), _ptr(a),
                                  int(b_add), int(a_add), _stream(stream)))

    def keygen_switch_key(self, kind, rotation, secret, a=None, e=None, seed=0, sigma=3.2, want_key=False,
                            stream=None):
        """Generate and install a rotation (WG_KEY_ROTATION), conjugation (WG_KEY_CONJ) or
        relinearisation (WG_KEY_RELIN) key on the device from the ternary secret (N int8 coefficients); a ([part][nq + np][N]) and e
        ([part][N]) given, or drawn from `seed` when None.  Returns the key as stored (flat uint64,
        wg_ctx_set_key layout) when want_key."""
        sec = np.ascontiguousarray(secret, dtype=np.int8)
        if sec.size != self.N:
            raise ValueError("secret must have N coefficients")
        ap = ep = None
        if a is not None:
            ap = np.ascontiguousarray(a, dtype=np.uint64)
            ep = np.ascontiguousarray(e, dtype=np.int64)
            parts = self.parts(self.nq - 1)
            if ap.size != parts * (self.nq + self.np_) * self.N or ep.size != parts * self.N:
                raise ValueError("mask / noise sizes do not match the key's parts and limbs")
        out = None
        if want_key:
            out = np.zeros(self.parts(self.nq - 1) * 2 * (self.nq + self.np_) * self.N, np.uint64)
        _check(lib().wg_keygen_switch_key(self.h, int(kind), int(rotation), sec.ctypes.data,
                                            None if ap is None else ap.ctypes.data,
                                            None if ep is None else ep.ctypes.data, int(seed) & (2**64 - 1),
                                            float(sigma), None if out is None else out.ctypes.data,
                                            _stream(stream)))
        return out

    def bundle_save(self, path, stages=()):
        """Write the context's keys and the given LtStage objects to `path` (wg_bundle_save)."""
        hs = np.ascontiguousarray([st.h.value for st in stages], dtype=np.uint64)
        _check(lib().wg_bundle_save(self.h, str(path).encode(), hs.ctypes.data if len(stages) else None, len(stages)))

    def bundle_load(self, path, max_stages=64):
        """Install the keys of a bundle file and return its stages as LtStage objects
        (wg_bundle_load)."""
        hs = (C.c_void_p * max_stages)()
        n = C.c_size_t()
        _check(lib().wg_bundle_load(self.h, str(path).encode(), hs, max_stages, C.byref(n)))
        return [LtStage.from_handle(self, C.c_void_p(hs[i])) for i in range(n.value)]

    def decrypt_decode(self, level, scales, cts, secret, stream=None):
        """Decrypt and decode on the device (wg_decrypt_decode): cts = [(b, a)] device tensors at
        `level` with scales[k]; returns the complex slots as a [count][N/2] array."""
        arr = lambda ts: np.ascontiguousarray([_ptr(t) for t in ts], dtype=np.uint64)
        pb, pa = arr([x[0] for x in cts]), arr([x[1] for x in cts])
        sc = np.ascontiguousarray(scales, dtype=np.float64)
        sec = np.ascontiguousarray(secret, dtype=np.int8)
        re = np.zeros((len(cts), self.N // 2))
        im = np.zeros((len(cts), self.N // 2))
        _check(lib().wg_decrypt_decode(self.h, len(cts), int(level), sc.ctypes.data, pb.ctypes.data, pa.ctypes.data,
                                       None, sec.ctypes.data, re.ctypes.data, im.ctypes.data, _stream(stream)))
        return re + 1j * im

    def encode_slots_device(self, limbs, scale, re, im, outs, eval_form=False, stream=None):
        """CKKS encoding on the device (wg_encode_slots_device) of slot vectors re / im ([count][N/2]
        float64) into outs (device tensors of limbs * N words)."""
        arr = lambda ts: np.ascontiguousarray([_ptr(t) for t in ts], dtype=np.uint64)
        r = np.ascontiguousarray(re, dtype=np.float64)
        i = np.ascontiguousarray(im, dtype=np.float64)
        ob = arr(outs)
        if r.size != len(outs) * (self.N // 2) or i.size != r.size:
            raise ValueError("slot arrays must be [count][N/2]")
        _check(lib().wg_encode_slots_device(self.h, len(outs), int(limbs), float(scale), r.ctypes.data, i.ctypes.data,
                                     ob.ctypes.data, 1 if eval_form else 0, _stream(stream)))

    def encrypt_symmetric(self, level, pts, secret, outs, a=None, e=None, seed=0, sigma=3.2, stream=None):
        """Secret-key encryption of evaluation-form plaintexts (device tensors, level+1 limbs)
        into outs = [(b, a)] device tensors (wg_encrypt_symmetric); a ([count][level+1][N]) and
        e ([count][N]) given, or drawn from `seed`."""
        arr = lambda ts: np.ascontiguousarray([_ptr(t) for t in ts], dtype=np.uint64)
        pp, ob, oa = arr(pts), arr([x[0] for x in outs]), arr([x[1] for x in outs])
        sec = np.ascontiguousarray(secret, dtype=np.int8)
        ap = None if a is None else np.ascontiguousarray(a, dtype=np.uint64)
        ep = None if e is None else np.ascontiguousarray(e, dtype=np.int64)
        _check(lib().wg_encrypt_symmetric(self.h, len(pts), level, pp.ctypes.data, sec.ctypes.data,
                                          None if ap is None else ap.ctypes.data,
                                          None if ep is None else ep.ctypes.data, int(seed) & (2**64 - 1),
                                          float(sigma), ob.ctypes.data, oa.ctypes.data, _stream(stream)))

    def aes_walsh_encrypt_round_key_bits(self, params, expanded_key, active_blocks, secret, outs, seed=0, sigma=3.2,
                                         stream=None):
        """The Walsh AES's 1408 encrypted round-key bits on the device
        (wg_aes_walsh_encrypt_round_key_bits) into outs = [(b, a)] device tensors; returns
        (scales, levels)."""
        arr = lambda ts: np.ascontiguousarray([_ptr(t) for t in ts], dtype=np.uint64)
        ob, oa = arr([x[0] for x in outs]), arr([x[1] for x in outs])
        sec = np.ascontiguousarray(secret, dtype=np.int8)
        ek = np.frombuffer(bytes(expanded_key), dtype=np.uint8).copy()
        sc = np.zeros(1408, np.float64)
        lv = np.zeros(1408, np.uintp)
        _check(lib().wg_aes_walsh_encrypt_round_key_bits(self.h, C.byref(params), ek.ctypes.data, int(active_blocks),
                                                         sec.ctypes.data, int(seed) & (2**64 - 1), float(sigma),
                                                         ob.ctypes.data, oa.ctypes.data, sc.ctypes.data,
                                                         lv.ctypes.data, _stream(stream)))
        return sc, lv.astype(np.int64)

    def aes_xboot_encrypt_round_key_bits(self, params, expanded_key, first_round_key_level, secret, outs, seed=0,
                                         sigma=3.2, stream=None):
        """The XBOOT AES's 1408 encrypted round-key bits on the device
        (wg_aes_xboot_encrypt_round_key_bits) into outs = [(b, a)] device tensors; returns
        (scales, levels)."""
        arr = lambda ts: np.ascontiguousarray([_ptr(t) for t in ts], dtype=np.uint64)
        ob, oa = arr([x[0] for x in outs]), arr([x[1] for x in outs])
        sec = np.ascontiguousarray(secret, dtype=np.int8)
        ek = np.frombuffer(bytes(expanded_key), dtype=np.uint8).copy()
        sc = np.zeros(1408, np.float64)
        lv = np.zeros(1408, np.uintp)
        _check(lib().wg_aes_xboot_encrypt_round_key_bits(self.h, C.byref(params), ek.ctypes.data,
                                                         int(first_round_key_level), sec.ctypes.data,
                                                         int(seed) & (2**64 - 1), float(sigma), ob.ctypes.data,
                                                         oa.ctypes.data, sc.ctypes.data, lv.ctypes.data,
                                                         _stream(stream)))
        return sc, lv.astype(np.int64)

    def keygen_secret_switch(self, kind, source, target, a=None, e=None, seed=0, sigma=3.2, want_key=False,
                             stream=None):
        """Generate and install a bootstrapping secret switch on the device: WG_KEY_SPARSE_TO_DENSE
        (hybrid key, a [part][nq + np][N], e [part][N]) or WG_KEY_DENSE_TO_SPARSE (compact q0/p0
        key, a [1][2][N], e [1][N]) from `source` to `target` (N int8 ternary coefficients each).
        Returns the key as stored when want_key."""
        src = np.ascontiguousarray(source, dtype=np.int8)
        tgt = np.ascontiguousarray(target, dtype=np.int8)
        if src.size != self.N or tgt.size != self.N:
            raise ValueError("secrets must have N coefficients")
        compact = kind == WG_KEY_DENSE_TO_SPARSE
        parts = 1 if compact else self.parts(self.nq - 1)
        limbs = 2 if compact else self.nq + self.np_
        ap = ep = None
        if a is not None:
            ap = np.ascontiguousarray(a, dtype=np.uint64)
            ep = np.ascontiguousarray(e, dtype=np.int64)
            if ap.size != parts * limbs * self.N or ep.size != parts * self.N:
                raise ValueError("mask / noise sizes do not match the key's parts and limbs")
        out = np.zeros(parts * 2 * limbs * self.N, np.uint64) if want_key else None
        _check(lib().wg_keygen_secret_switch(self.h, int(kind), src.ctypes.data, tgt.ctypes.data,
                                             None if ap is None else ap.ctypes.data,
                                             None if ep is None else ep.ctypes.data, int(seed) & (2**64 - 1),
                                             float(sigma), None if out is None else out.ctypes.data,
                                             _stream(stream)))
        return out

    def rotate(self, level, b, a, rotation, stream=None):
        _check(lib().wg_rotate(self.h, level, _ptr(b), _ptr(a), int(rotation), _stream(stream)))

    def rotate_noalloc(self, level, b, a, rotation, stream=None):
        """Rotation whose scratch is the library's fixed 32 MiB static device array: no device
        allocation happens in the call (see wg_rotate_noalloc in include/walsh_gpu.h)."""
        _check(lib().wg_rotate_noalloc(self.h, level, _ptr(b), _ptr(a), int(rotation), _stream(stream)))

    def conjugate(self, level, b, a, stream=None):
        _check(lib().wg_conjugate(self.h, level, _ptr(b), _ptr(a), _stream(stream)))

    def rotate_many(self, level, b, a, rotations, out, stream=None):
        r = np.ascontiguousarray(rotations, dtype=np.int64)
        _check(lib().wg_rotate_many(self.h, level, _ptr(b), _ptr(a), r.ctypes.data, len(r), _ptr(out),
                                    _stream(stream)))

    def modraise(self, target_level, bs, as_, stream=None):
        """Raise level-0 ciphertexts (lists of device tensors holding target_level+1 limbs,
        limb 0 = q0 input) to target_level, in place."""
        arr = lambda ts: np.ascontiguousarray([_ptr(t) for t in ts], dtype=np.uint64)
        pb, pa = arr(bs), arr(as_)
        _check(lib().wg_modraise(self.h, len(pb), target_level, pb.ctypes.data, pa.ctypes.data, _stream(stream)))

    def dense_to_sparse(self, bs, as_, stream=None):
        """Level-0 dense-to-sparse switch (q0/p0 key), in place."""
        arr = lambda ts: np.ascontiguousarray([_ptr(t) for t in ts], dtype=np.uint64)
        pb, pa = arr(bs), arr(as_)
        _check(lib().wg_dense_to_sparse(self.h, len(pb), pb.ctypes.data, pa.ctypes.data, _stream(stream)))

    def sparse_to_dense(self, levels, bs, as_, stream=None):
        """Sparse-to-dense hybrid switch of ciphertext i at levels[i], in place."""
        arr = lambda ts: np.ascontiguousarray([_ptr(t) for t in ts], dtype=np.uint64)
        pb, pa = arr(bs), arr(as_)
        lv = np.ascontiguousarray(levels, dtype=np.uintp)
        _check(lib().wg_sparse_to_dense(self.h, len(pb), lv.ctypes.data, pb.ctypes.data, pa.ctypes.data,
                                        _stream(stream)))

    def evalchebyshev(self, level, scale, coeffs, bs, as_, out_bs, out_as, target_scale=0.0, default_scale=None,
                      stream=None):
        """Chebyshev series sum_k coeffs[k] T_k(x) of ciphertexts sharing level and scale (lists of
        device tensors); results into out_bs / out_as.  Returns (out_level, out_scale)."""
        arr = lambda ts: np.ascontiguousarray([_ptr(t) for t in ts], dtype=np.uint64)
        pb, pa, ob, oa = arr(bs), arr(as_), arr(out_bs), arr(out_as)
        cf = np.ascontiguousarray(coeffs, dtype=np.float64)
        lvl, sc = C.c_size_t(), C.c_double()
        _check(lib().wg_evalchebyshev(self.h, len(pb), level, float(scale), cf.ctypes.data, len(cf), float(target_scale),
                                      float(scale if default_scale is None else default_scale), pb.ctypes.data,
                                      pa.ctypes.data, ob.ctypes.data, oa.ctypes.data, C.byref(lvl), C.byref(sc),
                                      _stream(stream)))
        return lvl.value, sc.value

    def bootstrap_evalmod(self, params, s2c, c2s, coeffs, bs, as_, out0, out1, stream=None):
        """EvalMod bootstrap of packed ciphertexts (device tensors with room for depth+1 limbs):
        params a BootstrapParams, s2c / c2s lists of LtStage, out0 / out1 lists of (b, a) device
        tensors.  Returns (out_level, out_scale)."""
        arr = lambda ts: np.ascontiguousarray([_ptr(t) for t in ts], dtype=np.uint64)
        hs = lambda sts: np.ascontiguousarray([st.h.value for st in sts], dtype=np.uint64)
        ps, pc = hs(s2c), hs(c2s)
        pb, pa = arr(bs), arr(as_)
        o0b, o0a = arr([x[0] for x in out0]), arr([x[1] for x in out0])
        o1b, o1a = arr([x[0] for x in out1]), arr([x[1] for x in out1])
        cf = np.ascontiguousarray(coeffs, dtype=np.float64)
        lvl, sc = C.c_size_t(), C.c_double()
        _check(lib().wg_bootstrap_evalmod(self.h, C.byref(params), ps.ctypes.data, len(ps), pc.ctypes.data, len(pc),
                                          cf.ctypes.data, len(cf), len(pb), pb.ctypes.data, pa.ctypes.data,
                                          o0b.ctypes.data, o0a.ctypes.data, o1b.ctypes.data, o1a.ctypes.data,
                                          C.byref(lvl), C.byref(sc), _stream(stream)))
        return lvl.value, sc.value

    def walsh_sbox(self, params, s2c, c2s, coeffs, block_count, level, scale, bits, out_bits, stream=None):
        """Mask-packed Walsh S-box of len(bits) instances: bits[i] = 8 (b, a) device tensors of
        instance i; out_bits likewise (room for depth+1 limbs).  Returns per-output-bit
        (levels, scales)."""
        count = len(bits)
        arr = lambda ts: np.ascontiguousarray([_ptr(t) for t in ts], dtype=np.uint64)
        hs = lambda sts: np.ascontiguousarray([st.h.value for st in sts], dtype=np.uint64)
        ib = arr([bits[i][k][0] for k in range(8) for i in range(count)])
        ia = arr([bits[i][k][1] for k in range(8) for i in range(count)])
        ob = arr([out_bits[i][k][0] for k in range(8) for i in range(count)])
        oa = arr([out_bits[i][k][1] for k in range(8) for i in range(count)])
        ps, pc = hs(s2c), hs(c2s)
        cf = np.ascontiguousarray(coeffs, dtype=np.float64)
        lv = np.zeros(8, np.uintp)
        sc = np.zeros(8, np.float64)
        _check(lib().wg_walsh_sbox(self.h, C.byref(params), ps.ctypes.data, len(ps), pc.ctypes.data, len(pc),
                                   cf.ctypes.data, len(cf), block_count, count, level, float(scale), ib.ctypes.data,
                                   ia.ctypes.data, ob.ctypes.data, oa.ctypes.data, lv.ctypes.data, sc.ctypes.data,
                                   _stream(stream)))
        return [int(x) for x in lv], [float(x) for x in sc]

    def xboot_sbox(self, level, scale, bits, outs):
        """The XBOOT S-box on instances of 8 bit ciphertexts: bits[i][k] = (b, a) device tensors
        at `level`; outs[i][k] receive the outputs.  Returns (levels, scales) of the 8 bits."""
        count = len(bits)
        flat = lambda sel, xs: np.ascontiguousarray([_ptr(xs[i][k][sel]) for k in range(8) for i in range(count)],
                                                    dtype=np.uint64)
        ib, ia, ob, oa = flat(0, bits), flat(1, bits), flat(0, outs), flat(1, outs)
        lv = np.zeros(8, np.uintp)
        sc = np.zeros(8, np.float64)
        _check(lib().wg_xboot_sbox(self.h, count, level, float(scale), ib.ctypes.data, ia.ctypes.data, ob.ctypes.data,
                                   oa.ctypes.data, lv.ctypes.data, sc.ctypes.data, _stream(None)))
        return [int(x) for x in lv], [float(x) for x in sc]

    def aes_ctr_walsh(self, params, s2c, s2c_x2, c2s, coeffs, packing_block_count, packed_segment_count, key_bits,
                      key_scales, key_level, counters, ciphertexts, active_blocks, out_bits, stream=None, plain=False):
        """Homomorphic AES-128-CTR on lazy bits: key_bits = 1408 (b, a) device tensors, counters /
        ciphertexts = bytes of 2 * active_blocks blocks, out_bits = 128 (b, a) device tensors.
        Returns (levels, scales) of the 128 output bits."""
        arr = lambda ts: np.ascontiguousarray([_ptr(t) for t in ts], dtype=np.uint64)
        hs = lambda sts: np.ascontiguousarray([st.h.value for st in sts], dtype=np.uint64)
        kb, ka = arr([x[0] for x in key_bits]), arr([x[1] for x in key_bits])
        ob, oa = arr([x[0] for x in out_bits]), arr([x[1] for x in out_bits])
        ps, ps2, pc = hs(s2c), hs(s2c_x2), hs(c2s)
        cf = np.ascontiguousarray(coeffs, dtype=np.float64)
        ks = np.ascontiguousarray(key_scales, dtype=np.float64)
        lv = np.zeros(128, np.uintp)
        sc = np.zeros(128, np.float64)
        fn = lib().wg_aes_ctr_walsh_plain if plain else lib().wg_aes_ctr_walsh
        _check(fn(self.h, C.byref(params), ps.ctypes.data, len(ps), ps2.ctypes.data, len(ps2), pc.ctypes.data,
                  len(pc), cf.ctypes.data, len(cf), packing_block_count, packed_segment_count, kb.ctypes.data,
                  ka.ctypes.data, ks.ctypes.data, key_level, bytes(counters), bytes(ciphertexts), active_blocks,
                  ob.ctypes.data, oa.ctypes.data, lv.ctypes.data, sc.ctypes.data, _stream(stream)))
        return [int(x) for x in lv], [float(x) for x in sc]

    def bootstrap_pair(self, params, s2c, c2s, coeffs, scale, pairs, stream=None):
        """XBOOT pair bootstraps: pairs = [((b0, a0), (b1, a1))] device tensors at level
        s2c_depth with room for depth+1 limbs, every first ciphertext at `scale`; the results
        overwrite them.  Returns (out_level, out_scale)."""
        arr = lambda ts: np.ascontiguousarray([_ptr(t) for t in ts], dtype=np.uint64)
        hs = lambda sts: np.ascontiguousarray([st.h.value for st in sts], dtype=np.uint64)
        ps, pc = hs(s2c), hs(c2s)
        b0, a0 = arr([x[0][0] for x in pairs]), arr([x[0][1] for x in pairs])
        b1, a1 = arr([x[1][0] for x in pairs]), arr([x[1][1] for x in pairs])
        cf = np.ascontiguousarray(coeffs, dtype=np.float64)
        lvl, sc = C.c_size_t(), C.c_double()
        _check(lib().wg_bootstrap_pair(self.h, C.byref(params), ps.ctypes.data, len(ps), pc.ctypes.data, len(pc),
                                       cf.ctypes.data, len(cf), len(pairs), float(scale), b0.ctypes.data,
                                       a0.ctypes.data, b1.ctypes.data, a1.ctypes.data, C.byref(lvl), C.byref(sc),
                                       _stream(stream)))
        return lvl.value, sc.value

    def aes_ctr_xboot(self, params, s2c, c2s, coeffs, key_bits, key_scales, key_levels, counters, ciphertexts,
                      blocks, out_bits, stream=None):
        """Homomorphic AES-128-CTR with the XBOOT S-box: key_bits = 1408 (b, a) device tensors at
        key_levels, counters / ciphertexts = bytes of `blocks` blocks, out_bits = 128 (b, a)
        device tensors with room for depth+1 limbs.  Returns (levels, scales) of the outputs."""
        arr = lambda ts: np.ascontiguousarray([_ptr(t) for t in ts], dtype=np.uint64)
        hs = lambda sts: np.ascontiguousarray([st.h.value for st in sts], dtype=np.uint64)
        kb, ka = arr([x[0] for x in key_bits]), arr([x[1] for x in key_bits])
        ob, oa = arr([x[0] for x in out_bits]), arr([x[1] for x in out_bits])
        ps, pc = hs(s2c), hs(c2s)
        cf = np.ascontiguousarray(coeffs, dtype=np.float64)
        ks = np.ascontiguousarray(key_scales, dtype=np.float64)
        kl = np.ascontiguousarray(key_levels, dtype=np.uintp)
        lv = np.zeros(128, np.uintp)
        sc = np.zeros(128, np.float64)
        _check(lib().wg_aes_ctr_xboot(self.h, C.byref(params), ps.ctypes.data, len(ps), pc.ctypes.data, len(pc),
                                      cf.ctypes.data, len(cf), kb.ctypes.data, ka.ctypes.data, ks.ctypes.data,
                                      kl.ctypes.data, bytes(counters), bytes(ciphertexts), blocks, ob.ctypes.data,
                                      oa.ctypes.data, lv.ctypes.data, sc.ctypes.data, _stream(stream)))
        return [int(x) for x in lv], [float(x) for x in sc]

    def xboot_initial_state(self, params, key_bits, key_scales, key_levels, counters, blocks, out_bits, stream=None):
        """The XBOOT AES's initial public XOR (wg_xboot_initial_state) from 128 round-0 key bits:
        returns (level, scales) of the 128 state bits written to out_bits."""
        arr = lambda ts: np.ascontiguousarray([_ptr(t) for t in ts], dtype=np.uint64)
        kb, ka = arr([x[0] for x in key_bits]), arr([x[1] for x in key_bits])
        ob, oa = arr([x[0] for x in out_bits]), arr([x[1] for x in out_bits])
        ks = np.ascontiguousarray(key_scales, dtype=np.float64)
        kl = np.ascontiguousarray(key_levels, dtype=np.uintp)
        lvl = C.c_size_t()
        sc = np.zeros(128, np.float64)
        _check(lib().wg_xboot_initial_state(self.h, C.byref(params), kb.ctypes.data, ka.ctypes.data, ks.ctypes.data,
                                            kl.ctypes.data, bytes(counters), blocks, ob.ctypes.data, oa.ctypes.data,
                                            C.byref(lvl), sc.ctypes.data, _stream(stream)))
        return lvl.value, [float(x) for x in sc]

    def xboot_linear_layer(self, level, in_scales, in_bits, key_bits, key_levels, mix, out_bits, stream=None):
        """ShiftRows + MixColumns (when mix) + AddRoundKey of the XBOOT AES
        (wg_xboot_linear_layer); returns the 128 output scales."""
        arr = lambda ts: np.ascontiguousarray([_ptr(t) for t in ts], dtype=np.uint64)
        ib, ia = arr([x[0] for x in in_bits]), arr([x[1] for x in in_bits])
        kb, ka = arr([x[0] for x in key_bits]), arr([x[1] for x in key_bits])
        ob, oa = arr([x[0] for x in out_bits]), arr([x[1] for x in out_bits])
        isc = np.ascontiguousarray(in_scales, dtype=np.float64)
        kl = np.ascontiguousarray(key_levels, dtype=np.uintp)
        sc = np.zeros(128, np.float64)
        _check(lib().wg_xboot_linear_layer(self.h, level, isc.ctypes.data, ib.ctypes.data, ia.ctypes.data,
                                           kb.ctypes.data, ka.ctypes.data, kl.ctypes.data, 1 if mix else 0,
                                           ob.ctypes.data, oa.ctypes.data, sc.ctypes.data, _stream(stream)))
        return [float(x) for x in sc]

    def mul(self, level, b1, a1, b2, a2, c2, stream=None):
        _check(lib().wg_mul(self.h, level, _ptr(b1), _ptr(a1), _ptr(b2), _ptr(a2), _ptr(c2), _stream(stream)))

    def relin(self, level, c0, c1, c2, stream=None):
        _check(lib().wg_relin(self.h, level, _ptr(c0), _ptr(c1), _ptr(c2), _stream(stream)))

    def rescale(self, level, polys, npolys=1, stride=0, stream=None):
        _check(lib().wg_rescale(self.h, level, _ptr(polys), npolys, stride, _stream(stream)))

    def add(self, level, x, y, npolys=1, stride=0, stream=None):
        _check(lib().wg_add(self.h, level, _ptr(x), _ptr(y), npolys, stride, _stream(stream)))

    def sub(self, level, x, y, npolys=1, stride=0, stream=None):
        _check(lib().wg_sub(self.h, level, _ptr(x), _ptr(y), npolys, stride, _stream(stream)))

    def batch_mul_relin_rescale_rotate(self, levels, xb, xa, yb, ya, rots, stream=None, plain=False):
        """mul + relin + rescale + rotate per ciphertext; batched launches, or op by op with
        plain=True (the per-operation path)."""
        n = len(levels)
        lv = np.ascontiguousarray(levels, dtype=np.uintp)
        arr = lambda ts: np.ascontiguousarray([_ptr(t) for t in ts], dtype=np.uint64)
        pxb, pxa, pyb, pya = arr(xb), arr(xa), arr(yb), arr(ya)
        r = np.ascontiguousarray(rots, dtype=np.int64)
        fn = lib().wg_sequence_mul_relin_rescale_rotate if plain else lib().wg_batch_mul_relin_rescale_rotate
        _check(fn(self.h, n, lv.ctypes.data, pxb.ctypes.data, pxa.ctypes.data, pyb.ctypes.data, pya.ctypes.data,
                  r.ctypes.data, _stream(stream)))
