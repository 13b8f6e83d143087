"""The integer arithmetic of the modular scheme, checked on the CPU (no GPU):
the residue pass's FP64 expressions, the GEMM epilogue's reduction of INT32
sums, and the margin the reconstruction's quotient estimate needs.

Residue pass, with exact rational arithmetic: for integers |a'| <= 2^53,

  h = RN(a' 2^-27 + M) - M,  l = a' - h 2^27           (M = 1.5 2^52)
  yb = h (2^27 mod p) + l + M                          (y = yb - M)
  qm = RN(y RN(1/p) + M),  q = qm - M,  r = y - q p

gives the unique representative of a' mod p in [-(p-1)/2, (p-1)/2] for every
odd modulus of the list, and every intermediate is exact in FP64 (|h|, |l| <=
2^26, |y| < 2^35).  RN is round-to-nearest-even, which Python's float() of a
Fraction performs exactly.  The device kernel evaluates the same expressions
with FMAs (single roundings of the exact values written here) and forms r in
32-bit integers from the low words of the doubles yb and qm:
(lo(yb) - lo(qm) p) mod 2^32, read as a signed word."""
from fractions import Fraction

import numpy as np
import pytest

MODULI = [256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193, 191, 181]
MAGIC = 6755399441055744.0          # 1.5 2^52


def rn(x):
    """Round an exact rational to the nearest double (ties to even)."""
    return float(x)


def residue(a, p):
    assert abs(a) <= 2 ** 53
    h = rn(Fraction(a) * Fraction(2) ** -27 + Fraction(MAGIC)) - MAGIC   # exact subtraction
    h = int(h)
    l = a - h * 2 ** 27
    assert abs(h) <= 2 ** 26 and abs(l) <= 2 ** 26
    c27 = (2 ** 27) % p
    y = h * c27 + l
    assert abs(y) < 2 ** 35
    inv = rn(Fraction(1, p))
    yb = rn(Fraction(y) + Fraction(MAGIC))
    assert yb - MAGIC == y                                  # exact
    qm = rn(Fraction(y) * Fraction(inv) + Fraction(MAGIC))
    q = int(qm - MAGIC)
    r = y - q * p
    # the device's integer form: low words of yb and qm, arithmetic mod 2^32
    rw = (low_word(yb) - low_word(qm) * p) % 2 ** 32
    assert (rw - 2 ** 32 if rw >= 2 ** 31 else rw) == r
    return r


def low_word(v):
    """The low 32 bits of the IEEE bit pattern of the double v."""
    return int(np.array([v], dtype=np.float64).view(np.uint64)[0]) & 0xFFFFFFFF


def cases(seed, count):
    rng = np.random.default_rng(seed)
    out = [0, 1, -1, 2 ** 53, -(2 ** 53), 2 ** 53 - 1, 2 ** 27, -(2 ** 27), 2 ** 26, 2 ** 26 + 1,
           -(2 ** 26) - 1]
    for _ in range(count):
        e = int(rng.integers(0, 54))
        out.append(int(rng.integers(-(2 ** e), 2 ** e + 1)) if e < 63 else 0)
    return out


@pytest.mark.parametrize("p", [p for p in MODULI if p % 2 == 1])
def test_centred_residue_for_every_odd_modulus(p):
    half = (p - 1) // 2
    for a in cases(p, 1500):
        r = residue(a, p)
        assert -half <= r <= half, (a, p, r)
        assert (r - a) % p == 0, (a, p, r)


def test_near_half_integer_quotients():
    """Values of y whose y / p lies closest to a half-integer (the rounding
    decision of q): y = (2j + 1)(p - 1) / 2 and neighbours, across the y range."""
    for p in [p for p in MODULI if p % 2 == 1]:
        for j in (0, 1, 7, 2 ** 20, 2 ** 26 - 3):
            for d in (-2, -1, 0, 1, 2):
                a = (2 * j + 1) * (p - 1) // 2 + d
                for sgn in (1, -1):
                    r = residue(sgn * a, p)
                    assert -(p - 1) // 2 <= r <= (p - 1) // 2
                    assert (r - sgn * a) % p == 0


def test_modulus_256_is_the_low_byte():
    """Modulus 256: the signed low byte of l is a' mod 256 in [-128, 127]."""
    rng = np.random.default_rng(3)
    for _ in range(5000):
        a = int(rng.integers(-(2 ** 53), 2 ** 53))
        h = int(rn(Fraction(a) * Fraction(2) ** -27 + Fraction(MAGIC)) - MAGIC)
        l = a - h * 2 ** 27
        byte = l & 0xFF
        signed = byte - 256 if byte >= 128 else byte
        assert (signed - a) % 256 == 0 and -128 <= signed <= 127


def test_reconstruction_quotient_margin():
    """The reconstruction takes q = rint(S / M) from an FP64 estimate of S / M,
    off by less than 2^-38 (S < 18 * 256 * M).  It is the right quotient as
    long as |C'| / M stays that far below 1/2.  The integer width P the library
    picks (ca3dmm_crt_bits) keeps k 2^(2P) < M / 2 with a relative margin above
    2^-30 for every modulus count and depth: checked here in exact integers."""
    import ca3dmm_b200 as cb
    L = cb.lib()
    rng = np.random.default_rng(9)
    ks = sorted(set([1, 2, 3, 100, 1000, 4096, 8000, 8192, 32768, 65536, 131071, 131072] +
                    [int(x) for x in rng.integers(1, 131073, 300)]))
    for nmod in range(8, 19):
        M = 1
        for p in MODULI[:nmod]:
            M *= p
        for k in ks:
            P = L.ca3dmm_crt_bits(nmod, k)
            if P < 2:
                continue
            bound = k * 2 ** (2 * P)          # |C'| <= k 2^(2P)
            assert 2 * bound < M, (nmod, k, P)
            margin = Fraction(M - 2 * bound, 2 * M)
            assert margin > Fraction(1, 2 ** 30), (nmod, k, P, float(margin))
            if P < 53:                          # and P is the largest width that fits
                assert 2 * k * 2 ** (2 * (P + 1)) >= M or P + 1 > 53, (nmod, k, P)


def _mod_i32(v, p):
    """The GEMM epilogue's reduction of an INT32 sum v mod p, restated with
    32-bit unsigned arithmetic: y = h (2^16 mod p) + (v mod 2^16) + bias with
    h = v >> 16, q = umulhi(y, floor(2^32 / p)), r = y - q p folded once."""
    c16 = (1 << 16) % p
    bias = ((8650752 + p - 1) // p) * p
    mrec = (1 << 32) // p
    h = v >> 16                                   # arithmetic shift (numpy int64)
    y = (h * c16 + (v & 0xFFFF) + bias).astype(np.uint64)
    assert np.all(y < (1 << 25))
    q = (y * np.uint64(mrec)) >> np.uint64(32)
    r0 = (y - q * np.uint64(p)).astype(np.int64)
    r = np.where(r0 >= p, r0 - p, r0)
    return r


@pytest.mark.parametrize("p", MODULI)
def test_epilogue_reduction_of_int32_sums(p):
    """Every INT32 sum the modular GEMM can form (|v| <= k 128^2 < 2^31 for
    k <= 131072) reduces to v mod p in [0, p)."""
    rng = np.random.default_rng(p)
    lim = 131072 * 128 * 128
    v = np.concatenate([rng.integers(-lim, lim + 1, 200000),
                        np.array([0, 1, -1, lim, -lim, 2 ** 16, -(2 ** 16), 2 ** 16 - 1,
                                  -(2 ** 31) + 1, 2 ** 31 - 1])]).astype(np.int64)
    r = _mod_i32(v, p)
    assert np.all((r >= 0) & (r < p))
    assert np.all((r - v) % p == 0)
