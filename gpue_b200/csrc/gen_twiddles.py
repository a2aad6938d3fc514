"""Write twiddles.h: correctly rounded cos/sin(2*pi*m/R) for the small radices.

The in-register butterflies of the line FFT multiply by W_R^m = exp(-2 pi i m/R)
with compile-time constants.  This script evaluates the constants with
50-digit decimal arithmetic (Taylor series after reduction to [0, pi/4]) and
emits a constexpr lookup that nvcc folds when R and m are constants.

    python gpue_b200/csrc/gen_twiddles.py > gpue_b200/csrc/twiddles.h
"""

from decimal import Decimal, getcontext

getcontext().prec = 60
RADICES = [2, 3, 4, 5, 6, 8, 10, 12, 16, 20, 24, 32, 40, 48, 64]


def pi():
    # Machin: pi = 16 atan(1/5) - 4 atan(1/239)
    def atan_inv(x):
        x = Decimal(x)
        s, t, n, k = Decimal(0), 1 / x, 1, 0
        while True:
            term = t / n
            if term < Decimal(10) ** -58:
                break
            s += term if k % 2 == 0 else -term
            t /= x * x
            n += 2
            k += 1
        return s
    return 16 * atan_inv(5) - 4 * atan_inv(239)


PI = pi()


def sincos(a):
    s, c, term, i = Decimal(0), Decimal(0), Decimal(1), 0
    # cos: sum (-1)^k a^(2k)/(2k)!, sin: sum (-1)^k a^(2k+1)/(2k+1)!
    term_c, term_s = Decimal(1), a
    k = 0
    while abs(term_c) > Decimal(10) ** -58 or abs(term_s) > Decimal(10) ** -58:
        c += term_c
        s += term_s
        k += 1
        term_c = -term_c * a * a / ((2 * k - 1) * (2 * k))
        term_s = -term_s * a * a / ((2 * k) * (2 * k + 1))
    return s, c


def cos_sin_frac(m, R):
    """cos and sin of 2*pi*m/R using symmetry so the series argument stays small."""
    m %= R
    # reduce to the first octant via exact rational arithmetic on m/R
    from fractions import Fraction
    f = Fraction(m, R)  # angle = 2 pi f, f in [0,1)
    sign_s = 1
    if f > Fraction(1, 2):
        f = 1 - f
        sign_s = -1
    sign_c = 1
    if f > Fraction(1, 4):
        f = Fraction(1, 2) - f
        sign_c = -1
    swap = False
    if f > Fraction(1, 8):
        f = Fraction(1, 4) - f
        swap = True
    a = 2 * PI * Decimal(f.numerator) / Decimal(f.denominator)
    s, c = sincos(a)
    if swap:
        s, c = c, s
    return float(sign_c * c), float(sign_s * s)


def main():
    print("// Generated by gen_twiddles.py -- do not edit.")
    print("// tw_cos(R, m) = cos(2 pi m / R), tw_sin(R, m) = sin(2 pi m / R), correctly")
    print("// rounded to double; constexpr so constant arguments fold at compile time.")
    print("#pragma once")
    print()
    for name, idx in (("tw_cos", 0), ("tw_sin", 1)):
        print("__host__ __device__ constexpr double %s(int R, int m) {" % name)
        print("    m = ((m % R) + R) % R;")
        for R in RADICES:
            vals = [cos_sin_frac(m, R)[idx] for m in range(R)]
            body = " : ".join("m == %d ? %r" % (m, v) for m, v in enumerate(vals[:-1]))
            print("    if (R == %d) return %s : %r;" % (R, body, vals[-1]))
        print("    return 0.0;")
        print("}")
        print()


if __name__ == "__main__":
    main()
