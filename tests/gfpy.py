"""Independent pure-Python GF(256) / GF((2^8)^2) arithmetic for definitional
checks in tests (written from scrs/src/algebra/gf256.rs and gf65536.rs).
Kept separate from the C oracle so the two cross-check each other."""
import numpy as np

POLY_LOW = 0x1B  # gf256.rs:32
GEN = 0x03       # gf256.rs:39
DELTA = 0x20     # gf65536.rs:20
GEN16 = 0x0108   # gf65536.rs:26


def mul_xtime(a, b):
    acc = 0
    for i in range(8):
        if (b >> i) & 1:
            acc ^= a
        hi = a & 0x80
        a = (a << 1) & 0xFF
        if hi:
            a ^= POLY_LOW
    return acc


EXP = [0] * 255
LOG = [0] * 256
_v = 1
for _i in range(255):
    EXP[_i] = _v
    LOG[_v] = _i
    _v = mul_xtime(_v, GEN)

MUL = np.zeros((256, 256), dtype=np.uint8)
for _a in range(1, 256):
    for _b in range(1, 256):
        MUL[_a, _b] = EXP[(LOG[_a] + LOG[_b]) % 255]


def mul(a, b):
    return int(MUL[a, b])


def inv(a):
    return 0 if a == 0 else EXP[(255 - LOG[a]) % 255]


def mul16(x, y):
    a, b, c, d = x & 0xFF, x >> 8, y & 0xFF, y >> 8
    ac, bd = mul(a, c), mul(b, d)
    return (ac ^ mul(DELTA, bd)) | ((mul(a ^ b, c ^ d) ^ ac) << 8)


def square16(x):
    return mul16(x, x)


def inv16(x):
    a, b = x & 0xFF, x >> 8
    if x == 0:
        return 0
    norm = mul(a, a) ^ mul(a, b) ^ mul(DELTA, mul(b, b))
    ni = inv(norm)
    return mul(a ^ b, ni) | (mul(b, ni) << 8)


def pow16(x, e):
    r = 1
    while e:
        if e & 1:
            r = mul16(r, x)
        x = mul16(x, x)
        e >>= 1
    return r


def scale_bytes(row: np.ndarray, c: int) -> np.ndarray:
    """c * row over GF(256), bytewise."""
    return MUL[c][row]


def scale16_bytes(row: np.ndarray, c: int) -> np.ndarray:
    """c * row over interleaved GF((2^8)^2) elements [a, b]."""
    a = row[0::2]
    b = row[1::2]
    c0, c1 = c & 0xFF, c >> 8
    out = np.empty_like(row)
    out[0::2] = MUL[c0][a] ^ MUL[mul(DELTA, c1)][b]
    out[1::2] = MUL[c1][a] ^ MUL[c0 ^ c1][b]
    return out


def lcg_bytes(n, seed):
    """Deterministic test bytes (splitmix64 stream)."""
    x = np.uint64(seed)
    out = np.empty(n, dtype=np.uint8)
    with np.errstate(over="ignore"):
        i = 0
        while i < n:
            x = np.uint64(x + np.uint64(0x9E3779B97F4A7C15))
            z = x
            z = np.uint64((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9))
            z = np.uint64((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB))
            z = z ^ (z >> np.uint64(31))
            chunk = np.frombuffer(int(z).to_bytes(8, "little"), dtype=np.uint8)
            take = min(8, n - i)
            out[i:i + take] = chunk[:take]
            i += take
    return out


def rng_bytes(n, seed):
    return np.random.default_rng(seed).integers(0, 256, size=n, dtype=np.uint8)
