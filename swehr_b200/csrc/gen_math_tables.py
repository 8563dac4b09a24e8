"""Generate swehr_math_tables.h: the constant tables of the project's own
exp/log kernels (swehr_math.h).

Every value is a mathematical constant evaluated here at 80 significant
digits with Python's `decimal` and split into a double-double (hi, lo):
  * 2^(j/64), j = 0..63                        (exp reconstruction, Tang 1989)
  * log(1 + i/32), i = 0..32                   (log argument reduction)
  * ln2/64, 64/ln2, ln2, and the Taylor coefficients 1/n! and 2/(2n+1).

Run:  python swehr_b200/csrc/gen_math_tables.py > swehr_b200/csrc/swehr_math_tables.h
"""
from decimal import Decimal, getcontext

getcontext().prec = 80


def dd(v: Decimal):
    hi = float(v)
    lo = float(v - Decimal(hi))
    return hi, lo


def ln(v: Decimal) -> Decimal:
    return v.ln()


def fmt(x: float) -> str:
    return x.hex()


def main():
    two = Decimal(2)
    ln2 = ln(two)
    out = []
    out.append("/* Generated by gen_math_tables.py -- do not edit.  Double-double splits of")
    out.append(" * mathematical constants computed with 80-digit decimal arithmetic. */")
    out.append("#ifndef SWEHR_MATH_TABLES_H")
    out.append("#define SWEHR_MATH_TABLES_H")
    h, l = dd(ln2 / 64)
    out.append(f"#define SW_LN2N_HI {fmt(h)}")
    out.append(f"#define SW_LN2N_LO {fmt(l)}")
    out.append(f"#define SW_INVLN2N {fmt(float(64 / ln2))}")
    h, l = dd(ln2)
    out.append(f"#define SW_LN2_HI {fmt(h)}")
    out.append(f"#define SW_LN2_LO {fmt(l)}")
    fact = Decimal(1)
    for n in range(1, 9):
        fact *= n
        out.append(f"#define SW_INVFACT{n} {fmt(float(Decimal(1) / fact))}")
    for n in range(1, 8):
        out.append(f"#define SW_ATANH_C{2*n+1} {fmt(float(Decimal(2) / Decimal(2*n + 1)))}")
    out.append("SW_TABLE const double sw_exp2_hi[64] = {")
    his, los = [], []
    for j in range(64):
        v = (two ** (Decimal(j) / 64))
        h, l = dd(v)
        his.append(fmt(h))
        los.append(fmt(l))
    out.append("  " + ",\n  ".join(his) + "};")
    out.append("SW_TABLE const double sw_exp2_lo[64] = {")
    out.append("  " + ",\n  ".join(los) + "};")
    his, los = [], []
    for i in range(33):
        v = ln(Decimal(1) + Decimal(i) / 32)
        h, l = dd(v)
        his.append(fmt(h))
        los.append(fmt(l))
    out.append("SW_TABLE const double sw_logc_hi[33] = {")
    out.append("  " + ",\n  ".join(his) + "};")
    out.append("SW_TABLE const double sw_logc_lo[33] = {")
    out.append("  " + ",\n  ".join(los) + "};")
    out.append("#endif")
    print("\n".join(out))


if __name__ == "__main__":
    main()
