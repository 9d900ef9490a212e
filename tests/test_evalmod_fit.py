"""The library's EvalMod fit and K bound (host code, no device) against the reference's
binboot_han_ki_discrete_multi_interval_approximate (src/math/poly_approx.cpp:565-681) and
required_binboot_k_bound (src/math/binboot_k_bound.cpp:53-89), compiled from the reference's
own sources: the same coefficients bit for bit on every AES parameter set's fit and on extra
shapes (half-integer K, double-angle iterations, small radius, pruning), and the same K."""
import ctypes as C
import math

import numpy as np
import pytest

# (K, degree, double_angle, interval radius, validation points, prune threshold) of the AES
# presets (src/ckks/parameters/ckks_aes_params.hpp): walsh15's K is the sparse-secret bound
# below; the XBOOT sets fix K.
RADIUS = math.nextafter(0.25, 0.0)
XBOOT15 = (12, 120, 0, RADIUS, 64, 0.0)
XBOOT14 = (7, 60, 0, RADIUS, 64, 0.0)
EXTRA = [(4.5, 80, 0, 1.0 / 32.0, 64, 1e-10), (6, 70, 2, 0.125, 32, 1e-6), (3, 40, 1, 0.2, 16, 0.0)]


def _ref_fit(R, K, degree, da, radius, points, prune):
    R.ref_evalmod_fit.argtypes = [C.c_double, C.c_size_t, C.c_size_t, C.c_double, C.c_size_t, C.c_double,
                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    out = np.zeros(degree + 1, np.float64)
    n = C.c_size_t()
    err = C.c_double()
    iv = np.zeros(2, np.float64)
    rc = R.ref_evalmod_fit(float(K), degree, da, float(radius), points, float(prune), out.ctypes.data, C.byref(n),
                           C.byref(err), iv.ctypes.data)
    assert rc == 0
    return {"coeffs": out[: n.value], "max_error": err.value, "interval": (iv[0], iv[1])}


def _ref_k(R, n, h, log2_fail):
    R.ref_evalmod_k_bound.argtypes = [C.c_size_t, C.c_size_t, C.c_double, C.c_void_p]
    k = C.c_size_t()
    assert R.ref_evalmod_k_bound(n, h, float(log2_fail), C.byref(k)) == 0
    return k.value


def test_k_bound_matches_reference(wg, ref_mod):
    R = ref_mod.ref()
    for n, h, f in ((1 << 15, 32, -16.0), (1 << 15, 64, -40.0), (1 << 14, 16, -30.0), (1 << 16, 192, -128.0)):
        assert wg.evalmod_k_bound(n, h, f) == _ref_k(R, n, h, f), (n, h, f)


def _walsh15(wg):
    return (wg.evalmod_k_bound(1 << 15, 32, -16.0), 100, 0, RADIUS, 128, 1e-10)


@pytest.mark.parametrize("which", ["walsh15", "xboot15", "xboot14", "extra0", "extra1", "extra2"])
def test_fit_matches_reference_bit_for_bit(wg, ref_mod, which):
    shape = {"walsh15": None, "xboot15": XBOOT15, "xboot14": XBOOT14,
             "extra0": EXTRA[0], "extra1": EXTRA[1], "extra2": EXTRA[2]}[which]
    if shape is None:
        shape = _walsh15(wg)
    mine = wg.evalmod_fit(*shape)
    ref = _ref_fit(ref_mod.ref(), *shape)
    assert mine["coeffs"].size == ref["coeffs"].size
    assert (mine["coeffs"].view(np.uint64) == ref["coeffs"].view(np.uint64)).all()
    assert mine["interval"] == ref["interval"]
    assert mine["max_error"] == ref["max_error"]
    if not which.startswith("extra"):  # the preset fits are accurate; the extra shapes only test parity
        assert mine["max_error"] < 1e-3


def test_fit_rejects_invalid_shapes(wg):
    with pytest.raises(wg.InvalidArgument):
        wg.evalmod_fit(0.0, 10, 0, 0.1, 16, 0.0)
    with pytest.raises(wg.InvalidArgument):
        wg.evalmod_fit(3.3, 10, 0, 0.1, 16, 0.0)  # neither integer nor half-integer
    with pytest.raises(wg.InvalidArgument):
        wg.evalmod_fit(3, 10, 0, 0.25, 16, 0.0)  # radius must stay below 1/4
    with pytest.raises(wg.InvalidArgument):
        wg.evalmod_fit(3, 10, 0, 0.1, 1, 0.0)
