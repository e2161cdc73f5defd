"""Generate lg_log_table.h, the table of the FP64 Box-Muller logarithm.

The logarithm (log_unit_interval in lg_common.cuh) reduces u = 2^e f with f
in [sqrt(1/2), sqrt(2)) to one of 91 centres F_j = 1 + j/128, j = -37 .. 53,
and needs for each the double invF_j = RN(1 / F_j) and L_j = -ln(invF_j)
rounded to the nearest double (the logarithm of the tabulated reciprocal
itself, so that ln f = L_j + log1p(f invF_j - 1) holds exactly).  invF_j is
the correctly rounded quotient of two integers; L_j comes from a 50-digit
decimal logarithm, rounded once to double.  j = 0 gives invF = 1, L = 0.

Run: python legendre_b200/csrc/gen_log_table.py > legendre_b200/csrc/lg_log_table.h
"""
from decimal import Decimal, getcontext
from fractions import Fraction

J_MIN, J_MAX = -37, 53


def entries():
    getcontext().prec = 50
    out = []
    for j in range(J_MIN, J_MAX + 1):
        inv = float(Fraction(128, 128 + j))  # correctly rounded 128 / (128 + j)
        lj = float(-Decimal(inv).ln())       # Decimal(inv) is the double's exact value
        out.append((j, inv, lj))
    return out


def render() -> str:
    lines = [
        "// Generated by gen_log_table.py: centres F_j = 1 + j/128, j = %d .. %d," % (J_MIN, J_MAX),
        "// {RN(1/F_j), RN(-ln RN(1/F_j))} for the FP64 Box-Muller logarithm.",
        "#pragma once",
        "",
        "namespace lg {",
        "",
        "constexpr int kLogTableMin = %d;" % J_MIN,
        "constexpr int kLogTableSize = %d;" % (J_MAX - J_MIN + 1),
        "",
        "__device__ const double2 kLogTable[kLogTableSize] = {",
    ]
    for j, inv, lj in entries():
        lines.append("    {%s, %s},  // j = %d" % (inv.hex(), lj.hex(), j))
    lines += ["};", "", "}  // namespace lg", ""]
    return "\n".join(lines)


if __name__ == "__main__":
    print(render(), end="")
