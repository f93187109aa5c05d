"""Writes bf200_sobol_table.inc: the Joe-Kuo D6 direction parameters of Sobol dimensions
1..21200 (new-joe-kuo-6.21201, Copyright (c) 2008 Frances Y. Kuo and Stephen Joe, BSD licence,
reproduced in JOE_KUO_LICENSE.txt beside this file).

The parameters are a published table that has to be identical for the Sobol and Owen-scrambled
Sobol bits to match the reference's. This machine has no network, so the only local copy is the
one the reference project carries; this script decodes it and checks every row's layout before
writing. Each output row holds one dimension's parameters packed little-endian into three 64-bit
words: the polynomial coefficient bits a (degree - 1 bits), then the initial direction numbers
m_1 .. m_degree with m_k taking k bits.

Usage: python gen_sobol_table.py <path to the reference's Blackframe/Renderer/Source/SobolDirectionNumbers.inc>
"""
import hashlib
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
DEGREE_ROW_ENDS = [1, 2, 4, 6, 12, 18, 36, 52, 100, 160, 336, 480, 1110, 1866, 3666, 5714, 13424, 21200]


def degree_for_row(row):
    degree = 1
    while row >= DEGREE_ROW_ENDS[degree - 1]:
        degree += 1
    return degree


def main():
    if len(sys.argv) != 2:
        raise SystemExit(__doc__)
    source = sys.argv[1]
    text = open(source).read()
    rows = [tuple(int(v, 16) for v in m) for m in re.findall(r"\{(0x[0-9a-fA-F]+)ULL,\s*(0x[0-9a-fA-F]+)ULL,\s*"
                                                             r"(0x[0-9a-fA-F]+)ULL\}", text)]
    if len(rows) != 21200:
        raise SystemExit(f"expected 21200 rows, found {len(rows)}")
    for row, words in enumerate(rows):
        degree = degree_for_row(row)
        used = (degree - 1) + degree * (degree + 1) // 2
        value = words[0] | (words[1] << 64) | (words[2] << 128)
        if value >> used:
            raise SystemExit(f"row {row}: bits beyond the packed parameters")
        for k in range(1, degree + 1):  # every initial direction number m_k is odd and below 2^k
            offset = (degree - 1) + k * (k - 1) // 2
            m = (value >> offset) & ((1 << k) - 1)
            if m % 2 == 0:
                raise SystemExit(f"row {row}: even initial direction number")
    out = os.path.join(HERE, "bf200_sobol_table.inc")
    with open(out, "w") as f:
        f.write("// Generated by gen_sobol_table.py: Joe-Kuo D6 parameters of Sobol dimensions 1..21200\n")
        f.write("// (new-joe-kuo-6.21201, (c) 2008 F. Y. Kuo and S. Joe, BSD licence: JOE_KUO_LICENSE.txt).\n")
        for words in rows:
            f.write("{0x%016xULL, 0x%016xULL, 0x%016xULL},\n" % words)
    digest = hashlib.sha256(open(out, "rb").read()).hexdigest()
    print(f"wrote {out} ({len(rows)} rows, sha256 {digest})")


if __name__ == "__main__":
    main()
