"""Writes fx_math_consts.h, the constants of fx_math.h, from exact decimal arithmetic (Python's
decimal module at 80 digits): each constant is the given real number rounded to the stated number
of significant bits, printed as a C hexadecimal floating literal (exact).

    python femorax_b200/csrc/gen_fx_math_consts.py
"""
import decimal as dm
import math
import os

dm.getcontext().prec = 80
D = dm.Decimal
TWO = D(2)


def ln2():
    return TWO.ln()


def pi():
    # Machin: pi = 16 atan(1/5) - 4 atan(1/239)
    def atan_inv(n):
        x = D(1) / n
        x2 = x * x
        s, t, k = D(0), x, 0
        while True:
            term = t / (2 * k + 1)
            if term == 0 or abs(term) < D(10) ** -85:
                break
            s += term if k % 2 == 0 else -term
            t *= x2
            k += 1
        return s
    return 16 * atan_inv(5) - 4 * atan_inv(239)


def round_bits(v, bits):
    """v rounded to `bits` significant bits (round half to even): an exact double, as a Decimal."""
    if v == 0:
        return D(0)
    e = 0
    while TWO ** e > abs(v):
        e -= 1
    while TWO ** (e + 1) <= abs(v):
        e += 1
    n = int((v * TWO ** (bits - 1 - e)).to_integral_value(rounding=dm.ROUND_HALF_EVEN))
    f = math.ldexp(n, e - bits + 1)  # exact: |n| < 2^bits <= 2^53
    return D(f)


def lit(v):
    """A Decimal that is exactly a double, as a C hexadecimal literal."""
    f = float(v)
    assert D(f) == v, v
    return f.hex()


def dbl(v):
    return round_bits(v, 53)


def main():
    L2, PI = ln2(), pi()
    out = ["/* Constants of fx_math.h, written by gen_fx_math_consts.py (do not edit): each the stated",
           "   real number rounded to the stated number of significant bits. */",
           "#ifndef FX_MATH_CONSTS_H", "#define FX_MATH_CONSTS_H", ""]

    def emit(name, v, note):
        out.append(f"#define {name} {lit(v)} /* {note} */")

    # exp: x = k ln2/32 + r; ln2/32 in three parts of 36, 36 and 53 bits (k ln2/32 parts exact for |k| < 2^17)
    c = L2 / 32
    l1 = round_bits(c, 36)
    l2 = round_bits(c - l1, 36)
    l3 = dbl(c - l1 - l2)
    emit("FXM_INV_LN2_32", dbl(32 / L2), "32 / ln 2")
    emit("FXM_LN2_32_1", l1, "ln 2 / 32, first 36 bits")
    emit("FXM_LN2_32_2", l2, "ln 2 / 32, next 36 bits")
    emit("FXM_LN2_32_3", l3, "ln 2 / 32, the rest")
    for k in range(3, 8):
        f = D(1)
        for i in range(2, k + 1):
            f *= i
        emit(f"FXM_EXP_C{k}", dbl(1 / f), f"1/{k}!")
    hi, lo = [], []
    for j in range(32):
        v = TWO ** (D(j) / 32) if j else D(1)
        h = dbl(v)
        hi.append(lit(h))
        lo.append(lit(dbl(v - h)))
    out.append("/* 2^(j/32), j = 0..31, as double-double: high and low parts */")
    out.append("#define FXM_EXP2_HI_INIT " + ", ".join(hi))
    out.append("#define FXM_EXP2_LO_INIT " + ", ".join(lo))
    # log: e ln2 + log m; ln 2 in a 42-bit high part (e ln2_hi exact for |e| < 2^11) and the rest
    lh = round_bits(L2, 42)
    emit("FXM_LN2_HI", lh, "ln 2, first 42 bits")
    emit("FXM_LN2_LO", dbl(L2 - lh), "ln 2, the rest")
    emit("FXM_SQRT2", dbl(TWO.sqrt()), "sqrt 2")
    for k in range(1, 14):
        emit(f"FXM_LOG_A{k}", dbl(D(2) / (2 * k + 1)), f"2/{2 * k + 1}")
    # cos: x = k pi/2 + r; pi/2 in parts of 33, 33 and 53 bits (k parts exact for |k| < 2^20)
    p = PI / 2
    p1 = round_bits(p, 33)
    p2 = round_bits(p - p1, 33)
    p3 = dbl(p - p1 - p2)
    emit("FXM_TWO_OVER_PI", dbl(2 / PI), "2 / pi")
    emit("FXM_PIO2_1", p1, "pi / 2, first 33 bits")
    emit("FXM_PIO2_2", p2, "pi / 2, next 33 bits")
    emit("FXM_PIO2_3", p3, "pi / 2, the rest")
    fact = [D(1)]
    for i in range(1, 24):
        fact.append(fact[-1] * i)
    for k in range(2, 11):
        emit(f"FXM_COS_C{k}", dbl(D((-1) ** k) / fact[2 * k]), f"(-1)^{k}/{2 * k}!")
    for k in range(1, 10):
        emit(f"FXM_SIN_S{k}", dbl(D((-1) ** k) / fact[2 * k + 1]), f"(-1)^{k}/{2 * k + 1}!")
    c2 = dbl(D(1) / 24)
    emit("FXM_COS_C2_LO", dbl(D(1) / 24 - c2), "1/24 - FXM_COS_C2")
    s1 = dbl(D(-1) / 6)
    emit("FXM_SIN_S1_LO", dbl(D(-1) / 6 - s1), "-1/6 - FXM_SIN_S1")
    out += ["", "#endif", ""]
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "fx_math_consts.h"), "w") as f:
        f.write("\n".join(out))


if __name__ == "__main__":
    main()
