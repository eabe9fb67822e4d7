"""Generates the reduction table of ln_dd.h (run: python gen_ln_table.py).

For m in [sqrt(1/2), sqrt(2)) the table splits [A, A + 183/256) into
intervals i of width 1/256 starting at A + i/256, with A = 359/512 chosen
so that interval 76 is centred on 1.  Entry i holds c_i = RN(1 / centre_i)
(exactly 1 for interval 76) and -ln(c_i) as a double-double, each rounded
from a 60-digit decimal evaluation, so ln m = ln(m * c_i) - ln(c_i) with
|m * c_i - 1| < 2^-8.4.
"""
from decimal import Decimal, getcontext
from fractions import Fraction

getcontext().prec = 60

A = Fraction(359, 512)
N = 183
CENTRE_ONE = 76


def dd(x: Decimal):
    hi = float(x)
    lo = float(x - Decimal(hi))
    return hi, lo


def table():
    rows = []
    for i in range(N):
        centre = A + Fraction(2 * i + 1, 512)
        c = 1.0 if i == CENTRE_ONE else float(1 / centre)
        if i == CENTRE_ONE:
            assert centre == 1
        minus_ln_c = -Decimal(c).ln() if c != 1.0 else Decimal(0)
        rows.append((c, *dd(minus_ln_c)))
    return rows


def main():
    rows = table()
    print("/* generated by gen_ln_table.py: c_i, -ln(c_i) hi, lo */")
    print("#define NECSIM_LN_TABLE_N %d" % N)
    for name, col in (("C", 0), ("LHI", 1), ("LLO", 2)):
        print("#define NECSIM_LN_TABLE_%s \\" % name)
        vals = [rows[i][col].hex() for i in range(N)]
        lines = []
        for j in range(0, N, 4):
            lines.append("    " + ", ".join(vals[j:j + 4]))
        print("    {" + (", \\\n".join(lines)).strip() + "}")


if __name__ == "__main__":
    main()
