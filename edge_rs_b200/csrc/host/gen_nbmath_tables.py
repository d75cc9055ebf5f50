"""Writes nbmath_tables.inc: the tables of the table-driven exp and log in
nbmath.hpp (Tang's method: P. T. P. Tang, "Table-driven implementation of the
exponential function in IEEE floating-point arithmetic", ACM TOMS 15(2), 1989,
and "... of the logarithm function ...", ACM TOMS 16(4), 1990).

Every entry is computed in 60-digit decimal arithmetic and rounded once to the
nearest double (Python's float(Decimal) rounds correctly), so the tables do
not depend on any platform's libm.

exp: T[j] = 2^(j/256), j = 0..255, as hi + lo.
log: for j = 0..256 the centre c_j = 1 + j/256, its reciprocal rounded to
     nine significant bits (inv_j = round(512 / c_j) / 512, so that
     m * inv_j - 1 is exact in one fused multiply-add for every mantissa m
     that maps to j), and -ln(inv_j) as hi + lo. j = 256 (c = 2, inv = 1/2)
     serves the mantissas just below 2 that round up to it; its -ln(inv) =
     ln 2 is split as the log's ln2_hi + ln2_lo.

Run: python gen_nbmath_tables.py > nbmath_tables.inc
"""
from decimal import Decimal, getcontext

getcontext().prec = 60
LN2 = Decimal(2).ln()


def hexd(x: float) -> str:
    return float.hex(x)


def split(v: Decimal):
    hi = float(v)
    lo = float(v - Decimal(hi))
    return hi, lo


def main():
    exp_rows = []
    for j in range(256):
        hi, lo = split((LN2 * j / 256).exp())
        exp_rows.append(f"    {{{hexd(hi)}, {hexd(lo)}}},  // 2^({j}/256)")
    log_rows, log_lo = [], []
    for j in range(257):
        c = Decimal(1) + Decimal(j) / 256
        k = int((Decimal(512) / c).to_integral_value())
        inv = Decimal(k) / 512
        assert float(inv) == k / 512
        hi, lo = split(-inv.ln())
        if j == 256:
            # -ln(1/2) = ln 2 split as the log's own ln2_hi (32 bits) + ln2_lo,
            # so that e ln2_hi + hi = (e + 1) ln2_hi stays exact and the
            # entry gives the double that rescaling m into [1/2, 1) would
            hi = float.fromhex("0x1.62e42fee00000p-1")
            lo = float(LN2 - Decimal(hi))
            assert lo == float.fromhex("0x1.a39ef35793c76p-33")
        log_rows.append(f"    {{{hexd(k / 512)}, {hexd(hi)}}},  // c = 1 + {j}/256, inv = {k}/512")
        log_lo.append(f"    {hexd(lo)},")
    out = ["// Generated by gen_nbmath_tables.py; do not edit. The brace-initializer",
           "// body of NbTableData (nbmath.hpp): exp pairs {hi, lo}, log pairs",
           "// {inv, hi}, log lo.",
           "{"]
    out += exp_rows
    out.append("},")
    out.append("{")
    out += log_rows
    out.append("},")
    out.append("{")
    out += log_lo
    out.append("},")
    print("\n".join(out))


if __name__ == "__main__":
    main()
