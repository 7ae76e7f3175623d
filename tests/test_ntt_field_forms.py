"""Field operations written as PTX carry sequences: the NTT's nt_sub, nt_add
(a subtraction of the negation), nt_canon, nt_reduce128 and the x 2^24 fold of gl_mul2_24 (ntt_field.cuh), and
the hash S-box's sqr_wide (gl64.cuh).  Each is replayed here instruction by
instruction with PTX's CC.CF semantics (add.cc / addc carry, sub.cc / subc
borrow, mad.lo.cc / madc.hi.cc, shf.l.wrap) and checked exactly against the
field (or the integer square) on random and edge-case operands.  The GPU
parity tests pin the compiled kernels' outputs; this pins the algebra of each
sequence."""

import random

import pytest

P = 0xFFFFFFFF00000001
M32 = 0xFFFFFFFF


class Flags:
    """The condition-code carry flag of a PTX instruction sequence (32-bit words)."""

    def __init__(self):
        self.cf = 0

    def add_cc(self, a, b):
        r = a + b
        self.cf = r >> 32
        return r & M32

    def addc_cc(self, a, b):
        r = a + b + self.cf
        self.cf = r >> 32
        return r & M32

    def addc(self, a, b):
        return (a + b + self.cf) & M32

    def sub_cc(self, a, b):
        r = a - b
        self.cf = int(r < 0)
        return r & M32

    def subc_cc(self, a, b):
        r = a - (b + self.cf)
        self.cf = int(r < 0)
        return r & M32

    def subc(self, a, b):
        return (a - (b + self.cf)) & M32

    def mad_lo_cc(self, a, b, c):
        r = ((a * b) & M32) + c
        self.cf = r >> 32
        return r & M32

    def madc_hi_cc(self, a, b, c):
        r = ((a * b) >> 32) + c + self.cf
        self.cf = r >> 32
        return r & M32


def halves(x):
    return x & M32, x >> 32


def mad_wide(a, b, c):
    return (a * b + c) % 2**64


def nt_sub(a, b):
    f = Flags()
    a0, a1 = halves(a)
    b0, b1 = halves(b)
    lo = f.sub_cc(a0, b0)
    hi = f.subc_cc(a1, b1)
    bw = f.subc(0, 0)
    lo = f.sub_cc(lo, bw)
    hi = f.subc(hi, 0)
    return (hi << 32) | lo


def nt_add(a, b):
    """nt_add: a - (p - b) through nt_sub (p - b is p itself when b = 0)."""
    return nt_sub(a, P - b)


def nt_canon(x):
    f = Flags()
    x0, x1 = halves(x)
    f.add_cc(x0, M32)
    f.addc_cc(x1, 0)
    k = f.addc(0, 0)
    return mad_wide(k, M32, x)


def nt_reduce128(l0, l1, h0, h1):
    f = Flags()
    r0 = f.sub_cc(l0, h1)
    r1 = f.subc_cc(l1, 0)
    b = f.subc(0, 0)
    r0 = f.sub_cc(r0, b)
    r1 = f.subc(r1, 0)
    r0 = f.mad_lo_cc(h0, M32, r0)
    r1 = f.madc_hi_cc(h0, M32, r1)
    k = f.addc(0, 0)
    return mad_wide(k, M32, (r1 << 32) | r0)


def nt_mul(a, b):
    v = a * b
    return nt_canon(nt_reduce128(v & M32, (v >> 32) & M32, (v >> 64) & M32, v >> 96))


def fold96(lo, h32):
    """lo + h32 * 2^64, as gl_mul2_24 forms x * 2^24 (canonical out)."""
    f = Flags()
    r0, r1 = halves(lo)
    r0 = f.mad_lo_cc(h32, M32, r0)
    r1 = f.madc_hi_cc(h32, M32, r1)
    k = f.addc(0, 0)
    return nt_canon(mad_wide(k, M32, (r1 << 32) | r0))


EDGES = [0, 1, 2, P - 1, P - 2, 0xFFFFFFFF, 0x100000000, 0xFFFFFFFF00000000, P // 2, 2**63, 0xFFFFFFFE00000001]


def test_edge_operands():
    for e1 in EDGES:
        for e2 in EDGES:
            a, b = e1 % P, e2 % P
            assert nt_sub(a, b) == (a - b) % P
            assert nt_add(a, b) == (a + b) % P
            assert nt_mul(a, b) == (a * b) % P


@pytest.mark.parametrize("seed", [1, 2])
def test_random_operands(seed):
    rng = random.Random(seed)
    for _ in range(20000):
        a, b = rng.randrange(P), rng.randrange(P)
        assert nt_sub(a, b) == (a - b) % P
        assert nt_add(a, b) == (a + b) % P
        assert nt_mul(a, b) == (a * b) % P
        x = rng.choice([rng.randrange(2**64), P + rng.randrange(2**32 - 1), rng.randrange(P)])
        assert nt_canon(x) == x % P
        v = rng.choice([rng.randrange(2**128), (2**64 - 1) ** 2, rng.randrange(2**64)])
        r = nt_reduce128(v & M32, (v >> 32) & M32, (v >> 64) & M32, v >> 96)
        assert r < 2**64 and r % P == v % P
        x = rng.randrange(P)
        assert fold96((x << 24) % 2**64, x >> 40) == x * 2**24 % P


def test_extreme_128_bit_inputs():
    for v in [(2**64 - 1) ** 2, 2**128 - 1, 0, 2**96, 2**96 - 1, P * (2**64 - 1)]:
        r = nt_reduce128(v & M32, (v >> 32) & M32, (v >> 64) & M32, v >> 96)
        assert r % P == v % P and nt_canon(r) == v % P


def sqr_wide(a):
    """gl64.cuh sqr_wide: a^2 from a0^2, a1^2 and the cross term a0 a1, doubled
    by a funnel shift (shf.l.wrap) and added once."""
    f = Flags()
    a0, a1 = halves(a)
    r0, r1 = (a0 * a0) & M32, (a0 * a0) >> 32
    r2, r3 = (a1 * a1) & M32, (a1 * a1) >> 32
    c0, c1 = (a0 * a1) & M32, (a0 * a1) >> 32
    c2 = c1 >> 31
    c1 = ((c1 << 1) | (c0 >> 31)) & M32  # shf.l.wrap.b32 c1, c0, c1, 1
    c0 = (c0 << 1) & M32
    r1 = f.add_cc(r1, c0)
    r2 = f.addc_cc(r2, c1)
    r3 = f.addc(r3, c2)
    return r0 | (r1 << 32) | (r2 << 64) | (r3 << 96)


def test_sqr_wide_is_the_exact_square():
    rnd = random.Random(11)
    edge = [0, 1, M32, M32 + 1, 2**63, 2**64 - 1, P - 1, P, 0x80000000, 0xFFFFFFFF80000000]
    for a in edge + [rnd.getrandbits(64) for _ in range(20000)]:
        assert sqr_wide(a) == a * a, hex(a)
