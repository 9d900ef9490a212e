"""Parameter sets used across the tests (bit sizes fed to the reference prime generator)."""

# config 1 of the benchmark description: N = 2^14, 16 Q limbs of ~50 bits, dnum = 4, P >= widest digit
CONFIG1 = dict(logN=14, q_bits=[50] * 16, p_bits=[50] * 4, dnum=4, h=192)

# the AESWalsh15 modulus chain as the reference's defaultQBits builds it
# (q0 36 | S2C 61 | mult 42, 42 | EvalMod 7 x 38 | C2S 50, 50), P = 4 x 61, dnum = 3
WALSH15 = dict(logN=15, q_bits=[36, 61, 42, 42] + [38] * 7 + [50, 50], p_bits=[61] * 4, dnum=3, h=256)

# small sets for fast parity sweeps
SMALL = [
    dict(logN=10, q_bits=[40, 45, 45, 45, 50], p_bits=[55, 55], dnum=3, h=64),
    dict(logN=11, q_bits=[36, 61, 42, 42, 38, 38], p_bits=[61, 61, 61], dnum=2, h=64),
    dict(logN=12, q_bits=[50] * 7, p_bits=[60, 60], dnum=4, h=64),
]
