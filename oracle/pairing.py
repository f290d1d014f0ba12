"""CPU restatement of libff's alt_bn128 reduced pairing (test infrastructure only).

The optimal ate pairing as libff computes it (third_party/.../libff/algebra/
curves/alt_bn128/alt_bn128_pairing.cpp: ate Miller loop over 6z + 2 with the
lines through pi(Q) and -pi^2(Q); final exponentiation whose last chunk is
Fuentes-Castaneda et al.'s multiple k = 2z(6z^2 + 3z + 1) of the exact hard
part, alt_bn128_pairing.cpp:152-224), restated with affine lines on the twist.
Two final exponentiations: final_exp raises to the whole exponent by
square-and-multiply, final_exp_chain follows libff's addition chain (the device
computes the chain); both give libff's value.

Tower: Fq2 = Fq[u]/(u^2 + 1), Fq6 = Fq2[v]/(v^3 - (9 + u)), Fq12 = Fq6[w]/(w^2 - v).
Elements are tuples of Python integers.  Pinned bit for bit against the
reference's own compiled libff (oracle/_ref, ref_reduced_pairing) by
tests/test_pairing_oracle.py.  Pure Python: a pairing takes about a second.
"""
import numpy as np

from oracle import P as q, R as r, fq_int, fq_mont

x = 4965661367192848881  # the BN parameter z
L = 6 * x + 2            # the ate loop count


def inv(a):
    return pow(a, q - 2, q)


# ---------------------------------------------------------------------------
# Fq2 = Fq[u]/(u^2 + 1)
# ---------------------------------------------------------------------------

XI = (9, 1)
Z2 = (0, 0)
O2 = (1, 0)


def f2add(a, b):
    return ((a[0] + b[0]) % q, (a[1] + b[1]) % q)


def f2sub(a, b):
    return ((a[0] - b[0]) % q, (a[1] - b[1]) % q)


def f2mul(a, b):
    return ((a[0] * b[0] - a[1] * b[1]) % q, (a[0] * b[1] + a[1] * b[0]) % q)


def f2neg(a):
    return ((-a[0]) % q, (-a[1]) % q)


def f2inv(a):
    n = inv((a[0] * a[0] + a[1] * a[1]) % q)
    return (a[0] * n % q, (-a[1]) * n % q)


def f2conj(a):
    return (a[0], (-a[1]) % q)


def f2s(a, k):
    """a times the integer k"""
    return (a[0] * k % q, a[1] * k % q)


# ---------------------------------------------------------------------------
# Fq6 = Fq2[v]/(v^3 - xi)
# ---------------------------------------------------------------------------

Z6 = (Z2, Z2, Z2)
O6 = (O2, Z2, Z2)


def f6add(a, b):
    return tuple(f2add(a[i], b[i]) for i in range(3))


def f6sub(a, b):
    return tuple(f2sub(a[i], b[i]) for i in range(3))


def f6neg(a):
    return tuple(f2neg(a[i]) for i in range(3))


def f6mul(a, b):
    a0, a1, a2 = a
    b0, b1, b2 = b
    c0 = f2add(f2mul(a0, b0), f2mul(XI, f2add(f2mul(a1, b2), f2mul(a2, b1))))
    c1 = f2add(f2add(f2mul(a0, b1), f2mul(a1, b0)), f2mul(XI, f2mul(a2, b2)))
    c2 = f2add(f2add(f2mul(a0, b2), f2mul(a1, b1)), f2mul(a2, b0))
    return (c0, c1, c2)


def f6mulv(a):
    """a v"""
    return (f2mul(XI, a[2]), a[0], a[1])


def f6inv(a):
    a0, a1, a2 = a
    t0 = f2sub(f2mul(a0, a0), f2mul(XI, f2mul(a1, a2)))
    t1 = f2sub(f2mul(XI, f2mul(a2, a2)), f2mul(a0, a1))
    t2 = f2sub(f2mul(a1, a1), f2mul(a0, a2))
    d = f2add(f2mul(a0, t0), f2mul(XI, f2add(f2mul(a2, t1), f2mul(a1, t2))))
    di = f2inv(d)
    return (f2mul(t0, di), f2mul(t1, di), f2mul(t2, di))


# ---------------------------------------------------------------------------
# Fq12 = Fq6[w]/(w^2 - v)
# ---------------------------------------------------------------------------

O12 = (O6, Z6)


def f12mul(a, b):
    a0, a1 = a
    b0, b1 = b
    return (f6add(f6mul(a0, b0), f6mulv(f6mul(a1, b1))), f6add(f6mul(a0, b1), f6mul(a1, b0)))


def f12conj(a):
    return (a[0], f6neg(a[1]))


def f12inv(a):
    a0, a1 = a
    t = f6inv(f6sub(f6mul(a0, a0), f6mulv(f6mul(a1, a1))))
    return (f6mul(a0, t), f6neg(f6mul(a1, t)))


def f12pow(a, e):
    res = O12
    for bit in bin(e)[2:]:
        res = f12mul(res, res)
        if bit == "1":
            res = f12mul(res, a)
    return res


# ---------------------------------------------------------------------------
# Miller loop
# ---------------------------------------------------------------------------

# Frobenius on the twist: pi(x, y) = (conj(x) FX1, conj(y) FY1) with
# FX1 = xi^((q-1)/3), FY1 = xi^((q-1)/2); pi^2(x, y) = (x FX2, y FY2) with
# FX2 = xi^((q^2-1)/3), FY2 = xi^((q^2-1)/2) = -1
FX1 = (0x2fb347984f7911f74c0bec3cf559b143b78cc310c2c3330c99e39557176f553d,
       0x16c9e55061ebae204ba4cc8bd75a079432ae2a1d0b7c9dce1665d51c640fcba2)
FY1 = (0x63cf305489af5dcdc5ec698b6e2f9b9dbaae0eda9c95998dc54014671a0135a,
       0x7c03cbcac41049a0704b5a7ec796f2b21807dc98fa25bd282d37f632623b0e3)
FX2 = (0x30644e72e131a0295e6dd9e7e0acccb0c28f069fbb966e3de4bd44e5607cfd48, 0)
FY2 = (q - 1, 0)


def line(lam, T, P):
    """The line of slope lam (on the twist) through T, at P: yP - lam xP w + (lam xT - yT) v w"""
    xP, yP = P
    c0 = ((yP % q, 0), Z2, Z2)
    c1 = (f2neg(f2s(lam, xP)), f2sub(f2mul(lam, T[0]), T[1]), Z2)
    return (c0, c1)


def _add_step(T, Q2, lam):
    x3 = f2sub(f2sub(f2mul(lam, lam), T[0]), Q2[0])
    return (x3, f2sub(f2mul(lam, f2sub(T[0], x3)), T[1]))


def miller(P, Q):
    """P = (x, y) on G1, Q = ((x0, x1), (y0, y1)) on the twist, both affine, finite."""
    f = O12
    T = Q
    for i in range(L.bit_length() - 2, -1, -1):
        lam = f2mul(f2s(f2mul(T[0], T[0]), 3), f2inv(f2s(T[1], 2)))
        f = f12mul(f12mul(f, f), line(lam, T, P))
        x3 = f2sub(f2mul(lam, lam), f2s(T[0], 2))
        T = (x3, f2sub(f2mul(lam, f2sub(T[0], x3)), T[1]))
        if (L >> i) & 1:
            lam = f2mul(f2sub(Q[1], T[1]), f2inv(f2sub(Q[0], T[0])))
            f = f12mul(f, line(lam, T, P))
            T = _add_step(T, Q, lam)
    Q1 = (f2mul(f2conj(Q[0]), FX1), f2mul(f2conj(Q[1]), FY1))
    nQ2 = (f2mul(Q[0], FX2), f2neg(f2mul(Q[1], FY2)))
    lam = f2mul(f2sub(Q1[1], T[1]), f2inv(f2sub(Q1[0], T[0])))
    f = f12mul(f, line(lam, T, P))
    T = _add_step(T, Q1, lam)
    lam = f2mul(f2sub(nQ2[1], T[1]), f2inv(f2sub(nQ2[0], T[0])))
    return f12mul(f, line(lam, T, P))


# ---------------------------------------------------------------------------
# final exponentiation
# ---------------------------------------------------------------------------

K_LIBFF = 2 * x * (6 * x * x + 3 * x + 1)
E_REST = (q**2 + 1) * K_LIBFF * ((q**4 - q**2 + 1) // r)


def final_exp(f):
    """f^((q^6 - 1)(q^2 + 1) k (q^4 - q^2 + 1)/r) by plain exponentiation"""
    f1 = f12mul(f12conj(f), f12inv(f))
    return f12pow(f1, E_REST)


def _f2pow(a, e):
    res = (1, 0)
    while e:
        if e & 1:
            res = f2mul(res, a)
        a = f2mul(a, a)
        e >>= 1
    return res


# GAMMA[k][m] = xi^(m (q^k - 1)/6): the factor of the coefficient of w^m under x^(q^k)
GAMMA = {k: [_f2pow(XI, m * (q**k - 1) // 6) for m in range(6)] for k in (1, 2, 3)}


def frobenius(xv, k):
    """x^(q^k); the coefficient of v^i w^j is that of w^(2i + j)"""
    def co(a, m):
        b = f2conj(a) if k % 2 else a
        return f2mul(b, GAMMA[k][m])
    c0, c1 = xv
    return (tuple(co(c0[i], 2 * i) for i in range(3)), tuple(co(c1[i], 2 * i + 1) for i in range(3)))


def exp_by_neg_z(xv):
    return f12conj(f12pow(xv, x))


def final_exp_chain(f):
    """the easy part, then libff's last chunk (alt_bn128_pairing.cpp:152-224)"""
    c = f12mul(f12conj(f), f12inv(f))
    elt = f12mul(frobenius(c, 2), c)
    A = exp_by_neg_z(elt)
    B = f12mul(A, A)
    D = f12mul(f12mul(B, B), B)
    E = exp_by_neg_z(D)
    G = exp_by_neg_z(f12mul(E, E))
    K = f12mul(f12mul(f12conj(G), E), f12conj(D))
    Lc = f12mul(K, B)
    N = f12mul(f12mul(K, E), elt)
    R = f12mul(frobenius(K, 2), f12mul(frobenius(Lc, 1), N))
    return f12mul(frobenius(f12mul(f12conj(elt), Lc), 3), R)


# ---------------------------------------------------------------------------
# libff layouts
# ---------------------------------------------------------------------------

def gt_limbs(g):
    """Fq12 -> alt_bn128_Fq12 Montgomery limbs (48 u64)"""
    vals = [c for c6 in g for c2 in c6 for c in c2]
    return np.concatenate([fq_mont(v) for v in vals])


def reduced_pairing_limbs(p_jac, q_jac):
    """libff layouts in (G1 12 u64 with Z = 1, G2 24 u64 with Z = 1), GT out (48 u64)."""
    P = (fq_int(p_jac[0:4]), fq_int(p_jac[4:8]))
    Q = ((fq_int(q_jac[0:4]), fq_int(q_jac[4:8])), (fq_int(q_jac[8:12]), fq_int(q_jac[12:16])))
    return gt_limbs(final_exp(miller(P, Q)))
