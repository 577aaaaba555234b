#!/usr/bin/env python3
"""Generate the standard-code data headers from the FeCl reference's tables.

The DVB-S2 LDPC parity-bit address tables (ETSI EN 302 307, Annexes B and C) and
the LTE turbo QPP interleaver parameters (3GPP TS 36.212, Table 5.1.3-3) are
standard data: a decoder for "the DVB-S2 code" or "the LTE interleaver" must use
exactly these numbers.  The reference ships them as C++ initialisers in
src/DvbS2.cpp:26-33 (lengths, rates, q parameters), src/DvbS2.cpp:35-1593
(addresses) and src/Lte3Gpp.cpp:26-217 (K, f1, f2).  This script parses those
initialisers and writes them out in this project's own flat layout:

  dvbs2_tables.h   one record per (n, rate): q, number of 360-bit groups and
                   the offset of its rows; one record per row: offset/length into
                   a flat address array.
  lte_qpp_table.h  188 (K, f1, f2) triples.

Run:  python3 extract_tables.py <reference-root>
"""
import os
import re
import sys


def _parse_braces(text):
    """Parse a nested {...} initialiser of unsigned integers into lists."""
    pos = 0
    toks = re.findall(r"\{|\}|[0-9]+(?:\.[0-9]+)?", text)

    def parse():
        nonlocal pos
        assert toks[pos] == "{"
        pos += 1
        out = []
        while toks[pos] != "}":
            if toks[pos] == "{":
                out.append(parse())
            else:
                out.append(toks[pos])
                pos += 1
        pos += 1
        return out

    return parse()


def _initialiser(src, name):
    m = re.search(re.escape(name) + r"\s*=\s*", src)
    if not m:
        raise SystemExit("initialiser %s not found" % name)
    start = src.index("{", m.end() - 1)
    depth = 0
    for i in range(start, len(src)):
        if src[i] == "{":
            depth += 1
        elif src[i] == "}":
            depth -= 1
            if depth == 0:
                return src[start:i + 1]
    raise SystemExit("unterminated initialiser %s" % name)


# Rates in the order the reference lists them (src/DvbS2.cpp:27-29), as fractions.
_RATES = [(1, 4), (1, 3), (2, 5), (1, 2), (3, 5), (2, 3), (3, 4), (4, 5), (5, 6), (8, 9), (9, 10)]


def dvbs2(ref_root):
    src = open(os.path.join(ref_root, "src", "DvbS2.cpp")).read()
    lengths = [int(x) for x in _parse_braces(_initialiser(src, "Ldpc::DvbS2::length_"))]
    params = _parse_braces(_initialiser(src, "Ldpc::DvbS2::parameter_"))
    index = _parse_braces(_initialiser(src, "Ldpc::DvbS2::index_"))
    codes, rows, addrs = [], [], []
    for li, n in enumerate(lengths):
        for ri, q in enumerate(params[li]):
            q = int(q)
            table = index[li][ri]
            codes.append((n, _RATES[ri][0], _RATES[ri][1], q, len(rows), len(table)))
            for row in table:
                rows.append((len(addrs), len(row)))
                addrs.extend(int(x) for x in row)
    return codes, rows, addrs


def lte(ref_root):
    src = open(os.path.join(ref_root, "src", "Lte3Gpp.cpp")).read()
    lengths = [int(x) for x in _parse_braces(_initialiser(src, "Turbo::Lte3Gpp::length_"))]
    params = [(int(a), int(b)) for a, b in _parse_braces(_initialiser(src, "Turbo::Lte3Gpp::parameter_"))]
    assert len(lengths) == len(params) == 188
    return [(k, f1, f2) for k, (f1, f2) in zip(lengths, params)]


def _wrap(values, per_line=12):
    vals = [str(v) for v in values]
    return ",\n".join("  " + ", ".join(vals[i:i + per_line]) for i in range(0, len(vals), per_line))


def main():
    if len(sys.argv) > 1:
        ref = sys.argv[1]
    elif os.environ.get("FECL_REFERENCE_DIR"):
        ref = os.environ["FECL_REFERENCE_DIR"]
    else:
        sys.exit("usage: extract_tables.py <reference source tree> (or set FECL_REFERENCE_DIR)")
    here = os.path.dirname(os.path.abspath(__file__))
    codes, rows, addrs = dvbs2(ref)
    with open(os.path.join(here, "dvbs2_tables.h"), "w") as f:
        f.write("/* Generated by extract_tables.py from the DVB-S2 address tables (ETSI EN 302 307\n"
                " * Annexes B, C) as listed in the reference's src/DvbS2.cpp.  Do not edit. */\n")
        f.write("#pragma once\n#include <stdint.h>\n\n")
        f.write("/* n, rate numerator, rate denominator, q, first row, number of 360-bit groups */\n")
        f.write("#define FECL_DVBS2_CODE_COUNT %d\n" % len(codes))
        f.write("static const uint32_t fecl_dvbs2_codes[FECL_DVBS2_CODE_COUNT][6] = {\n")
        f.write(",\n".join("  {%d, %d, %d, %d, %d, %d}" % c for c in codes))
        f.write("\n};\n\n/* offset into fecl_dvbs2_addr, number of addresses */\n")
        f.write("#define FECL_DVBS2_ROW_COUNT %d\n" % len(rows))
        f.write("static const uint32_t fecl_dvbs2_rows[FECL_DVBS2_ROW_COUNT][2] = {\n")
        f.write(",\n".join("  {%d, %d}" % r for r in rows))
        f.write("\n};\n\n#define FECL_DVBS2_ADDR_COUNT %d\n" % len(addrs))
        f.write("static const uint32_t fecl_dvbs2_addr[FECL_DVBS2_ADDR_COUNT] = {\n")
        f.write(_wrap(addrs))
        f.write("\n};\n")
    qpp = lte(ref)
    with open(os.path.join(here, "lte_qpp_table.h"), "w") as f:
        f.write("/* Generated by extract_tables.py from the LTE QPP interleaver parameters\n"
                " * (3GPP TS 36.212 Table 5.1.3-3) as listed in the reference's src/Lte3Gpp.cpp.\n"
                " * Do not edit. */\n")
        f.write("#pragma once\n#include <stdint.h>\n\n#define FECL_LTE_QPP_COUNT %d\n" % len(qpp))
        f.write("/* K, f1, f2 */\nstatic const uint32_t fecl_lte_qpp[FECL_LTE_QPP_COUNT][3] = {\n")
        f.write(",\n".join("  {%d, %d, %d}" % t for t in qpp))
        f.write("\n};\n")
    print("dvbs2: %d codes, %d rows, %d addresses; lte: %d sizes" % (len(codes), len(rows), len(addrs), len(qpp)))


if __name__ == "__main__":
    main()
