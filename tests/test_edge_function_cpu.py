"""The watertight test's edge-function fallback: a*b - c*d by Kahan's FMA
algorithm in single precision (trace.cuh diffOfProducts on the GPU, the
oracle's Tracer::diffOfProducts on the host, same operations). It replaced a
double-precision evaluation, so the GPU keeps FP64 to accumulation and the
environment CDF. What watertightness needs from it is checked here against
exact rational arithmetic:
  - the result is exactly zero when a*b == c*d (a ray through a shared edge
    or vertex is on the edge for both triangles);
  - otherwise its sign is the exact sign (a ray beside an edge is inside
    exactly one of the two triangles);
  - its error is at most 2 ulp of the exact value (Jeannerod, Louvet and
    Muller 2013), the bound the sign argument rests on.
Tolerance: sign and zero exact; magnitude within 2 * 2^-24 relative."""
from fractions import Fraction

import numpy as np

import oracle


def exact(a, b, c, d):
    return Fraction(float(a)) * Fraction(float(b)) - Fraction(float(c)) * Fraction(float(d))


def check(abcd):
    got = oracle.diff_of_products(abcd)
    for (a, b, c, d), r in zip(abcd, got):
        e = exact(a, b, c, d)
        if e == 0:
            assert r == 0.0, (a, b, c, d, r)
            continue
        assert (r > 0) == (e > 0) and r != 0.0, (a, b, c, d, r, float(e))
        assert abs(Fraction(float(r)) - e) <= Fraction(2, 1 << 24) * abs(e), (a, b, c, d, r, float(e))
    return got


def test_equal_products_give_exact_zero():
    rng = np.random.default_rng(3)
    u, v, w, z = (rng.integers(1, 4096, 4000).astype(np.float64) for _ in range(4))
    sgn = rng.choice([-1.0, 1.0], (4000, 2))
    scale = np.ldexp(1.0, rng.integers(-20, 20, (4000, 4)))
    # a*b = (u v)(w z) = (u w)(v z) = c*d, every factor exact in float32
    a = u * v * scale[:, 0] * sgn[:, 0]
    b = w * z * scale[:, 1] * sgn[:, 1]
    c = u * w * scale[:, 0] * sgn[:, 0]
    d = v * z * scale[:, 1] * sgn[:, 1]
    abcd = np.stack([a, b, c, d], 1).astype(np.float32)
    assert np.array_equal(abcd.astype(np.float64), np.stack([a, b, c, d], 1))
    got = check(abcd)
    assert np.all(got == 0.0)


def test_signs_near_cancellation_and_random():
    rng = np.random.default_rng(4)
    n = 3000
    a = rng.uniform(-2, 2, n).astype(np.float32)
    b = rng.uniform(-2, 2, n).astype(np.float32)
    # c*d within a few ulp of a*b: the plain float difference often rounds
    # to zero or the wrong sign here, the fallback must not
    steps = rng.integers(-3, 4, n)
    c = np.array([np.nextafter(x, np.float32(np.inf) if s > 0 else np.float32(-np.inf)) if s else x
                  for x, s in zip(a, steps)], np.float32)
    d = b.copy()
    check(np.stack([a, b, c, d], 1))
    check(rng.uniform(-1e3, 1e3, (n, 4)).astype(np.float32))


def test_edge_function_of_a_shared_edge_is_antisymmetric_in_sign():
    """The two triangles on a shared edge evaluate it with operands swapped
    (U of one is -U of the other): the signs are always opposite or both
    zero, which is what makes the test watertight."""
    rng = np.random.default_rng(5)
    p = rng.uniform(-1, 1, (5000, 4)).astype(np.float32)
    p[:2500, 2:] = p[:2500, :2] * np.float32(0.5)  # some exact zeros
    fwd = oracle.diff_of_products(p[:, [0, 3, 1, 2]])   # Cx*By - Cy*Bx
    rev = oracle.diff_of_products(p[:, [1, 2, 0, 3]])   # Cy*Bx - Cx*By
    assert np.array_equal(np.sign(fwd), -np.sign(rev))
