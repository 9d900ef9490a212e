"""Plain AES-128 for the tests: key expansion and block encryption restated from FIPS-197
(S-box from the GF(2^8) inverse and the affine map), used to check decrypted homomorphic
AES-CTR outputs."""


def _gmul(a, b):
    r = 0
    while b:
        if b & 1:
            r ^= a
        hi = a & 0x80
        a = (a << 1) & 0xFF
        if hi:
            a ^= 0x1B
        b >>= 1
    return r


def _sbox():
    s = []
    for x in range(256):
        inv = 0
        if x:
            r, p, e = 1, x, 254
            while e:
                if e & 1:
                    r = _gmul(r, p)
                p = _gmul(p, p)
                e >>= 1
            inv = r
        rot = lambda v, k: ((v << k) | (v >> (8 - k))) & 0xFF
        s.append(inv ^ rot(inv, 1) ^ rot(inv, 2) ^ rot(inv, 3) ^ rot(inv, 4) ^ 0x63)
    return s


SBOX = _sbox()


def expand_key(key):
    """176-byte expanded key of a 16-byte AES-128 key."""
    w = list(key)
    rcon = 1
    while len(w) < 176:
        t = w[-4:]
        if len(w) % 16 == 0:
            t = t[1:] + t[:1]
            t = [SBOX[b] for b in t]
            t[0] ^= rcon
            rcon = _gmul(rcon, 2)
        w += [w[-16 + i] ^ t[i] for i in range(4)]
    return bytes(w)


def encrypt_block(ek, block):
    s = [block[i] ^ ek[i] for i in range(16)]
    for rnd in range(1, 11):
        s = [SBOX[b] for b in s]
        s = [s[4 * ((c + r) % 4) + r] for c in range(4) for r in range(4)]
        if rnd < 10:
            out = []
            for c in range(4):
                a = s[4 * c:4 * c + 4]
                for r in range(4):
                    out.append(_gmul(a[r], 2) ^ _gmul(a[(r + 1) % 4], 3) ^ a[(r + 2) % 4] ^ a[(r + 3) % 4])
            s = out
        s = [s[i] ^ ek[16 * rnd + i] for i in range(16)]
    return bytes(s)
