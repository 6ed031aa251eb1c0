"""Generate dist_tables.h: the static 4-context frequency model of the PRZM
Mode 12 distance-code coder (Section 3 offsets).

The table is part of the PRZM bitstream format (a decoder holds the same
numbers), so it has to be identical to the reference's, value for value:
core/distance/distance.go:67-93 (StaticDistFreq4) and its C twin in
src/przm_dec.c.  This script reads the Go file of a reference checkout and
writes the numbers out as a C header; the header is committed, so neither a
build nor a test needs the reference checkout.

usage: python gen_dist_tables.py /path/to/przm-checkout > dist_tables.h
"""
import re
import sys


def main() -> None:
    if len(sys.argv) != 2:
        raise SystemExit("usage: python gen_dist_tables.py /path/to/przm-checkout > dist_tables.h")
    src = open(f"{sys.argv[1]}/core/distance/distance.go").read()
    start = src.index("{", src.index("var StaticDistFreq4"))
    stop = src.index("type distModel")
    nums = [int(x) for x in re.findall(r"\b\d+\b", src[start:stop])]
    if len(nums) != 4 * 64:
        raise SystemExit(f"expected 256 weights, found {len(nums)}")
    rows = [nums[c * 64:(c + 1) * 64] for c in range(4)]
    for c, row in enumerate(rows):
        if sum(row) != 4096 or min(row) < 1:
            raise SystemExit(f"context {c}: weights must be >= 1 and sum to 4096")
    out = [
        "/* Generated by gen_dist_tables.py -- do not edit.",
        " * Static per-context symbol weights (sum 4096 per context) of the PRZM",
        " * Mode 12 distance-code coder; identical to core/distance/distance.go:67-93",
        " * of the reference because they are part of the bitstream format. */",
        "#ifndef PRZM_DIST_TABLES_H",
        "#define PRZM_DIST_TABLES_H",
        "#include <stdint.h>",
        "static const uint16_t przm_dist_freq4[4][64] = {",
    ]
    for row in rows:
        out.append("  {")
        for i in range(0, 64, 16):
            out.append("    " + ", ".join(str(v) for v in row[i:i + 16]) + ",")
        out.append("  },")
    out += ["};", "#endif", ""]
    sys.stdout.write("\n".join(out))


if __name__ == "__main__":
    main()
