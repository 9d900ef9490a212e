"""The XBOOT S-box's integer coefficients (wg_xboot_sbox_coefficients): every output bit of the AES
S-box equals the sum of the coefficients of the monomials contained in the input (the Moebius
inversion of the bit's truth table), for all 256 inputs, and the table equals the reference's
(ckks_aes_ctr.cpp:258-278, through the harness) when the reference is built."""
import numpy as np

from aes_util import SBOX


def test_coefficients_reproduce_the_sbox(wg):
    cf = wg.xboot_sbox_coefficients()
    for x in range(256):
        subsets = [m for m in range(256) if m & x == m]
        for bit in range(8):
            assert int(cf[bit][subsets].sum()) == (SBOX[x] >> bit) & 1


def test_coefficients_match_the_reference(wg, ref_mod):
    assert (wg.xboot_sbox_coefficients() == ref_mod.RefXboot.coefficients()).all()
