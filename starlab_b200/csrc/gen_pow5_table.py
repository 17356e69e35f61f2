"""Writes pow5_table.h: 128-bit approximations of 5^q for q in [-342, 308],
the table of the Eisel-Lemire decimal-to-binary conversion (D. Lemire,
"Number parsing at a gigabyte per second", Software: Practice and
Experience 51(8), 2021; N. Mushtak and D. Lemire, "Fast number parsing
without fallback", SP&E 53(7), 2023) used by story_num.h.

Entry q is a 128-bit integer c with its top bit set:
  q >= 0: 5^q shifted left until bit 127 is its leading bit, then
          truncated to 128 bits;
  q < 0:  for z = bit length of 5^-q, c = floor(2^b / 5^-q) + 1 with
          b = z + 127 when q >= -27, else b = 2z + 128 and c truncated to
          its top 128 bits.
Run: python gen_pow5_table.py > pow5_table.h
"""

LO, HI = -342, 308


def entry(q):
    if q >= 0:
        c = 5 ** q
        while c < (1 << 127):
            c <<= 1
        while c >= (1 << 128):
            c >>= 1
        return c
    p = 5 ** -q
    z = p.bit_length()
    if q >= -27:
        return (1 << (z + 127)) // p + 1
    c = (1 << (2 * z + 128)) // p + 1
    while c >= (1 << 128):
        c >>= 1
    return c


def main():
    print("// pow5_table.h -- written by gen_pow5_table.py (see there); do not edit.")
    print("#pragma once")
    print("#define SN_POW5_MIN_Q (%d)" % LO)
    print("#define SN_POW5_MAX_Q %d" % HI)
    print("// {high 64 bits, low 64 bits} of entry q, at index 2 * (q - SN_POW5_MIN_Q)")
    print("#define SN_POW5_TABLE \\")
    print("    { \\")
    for q in range(LO, HI + 1):
        c = entry(q)
        assert (1 << 127) <= c < (1 << 128)
        print("        0x%016xull, 0x%016xull, /* %d */ \\" % (c >> 64, c & ((1 << 64) - 1), q))
    print("    }")


if __name__ == "__main__":
    main()
