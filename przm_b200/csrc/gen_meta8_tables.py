"""Generate meta8_tables.h: the static 8-context frequency model of the PRZM
Meta8 command-substream coder.

The table is part of the PRZM bitstream format (a decoder holds the same
numbers), so it has to be identical to the reference's, value for value:
core/commands/vans_meta_tables.go:7-154 (StaticMetaFreq8) and its C twin
src/vans_meta_tables.h.  This script reads the Go file of a reference
checkout and writes the numbers out as a C header; the header is committed,
so neither a build nor a test needs the reference checkout.

usage: python gen_meta8_tables.py /path/to/przm-checkout > meta8_tables.h
"""
import re
import sys


def main() -> None:
    if len(sys.argv) != 2:
        raise SystemExit("usage: python gen_meta8_tables.py /path/to/przm-checkout > meta8_tables.h")
    src = open(f"{sys.argv[1]}/core/commands/vans_meta_tables.go").read()
    start = src.index("{", src.index("StaticMetaFreq8"))
    stop = src.index("var staticMetaFreq8")
    nums = [int(x) for x in re.findall(r"\b\d+\b", src[start:stop])]
    if len(nums) != 8 * 256:
        raise SystemExit(f"expected 2048 weights, found {len(nums)}")
    rows = [nums[c * 256:(c + 1) * 256] for c in range(8)]
    for c, row in enumerate(rows):
        if sum(row) != 4096 or min(row) < 1:
            raise SystemExit(f"context {c}: weights must be >= 1 and sum to 4096")
    out = [
        "/* Generated by gen_meta8_tables.py -- do not edit.",
        " * Static per-context symbol weights (sum 4096 per context) of the PRZM",
        " * Meta8 bigram coder; identical to core/commands/vans_meta_tables.go:7-154",
        " * of the reference because they are part of the bitstream format. */",
        "#ifndef PRZM_META8_TABLES_H",
        "#define PRZM_META8_TABLES_H",
        "#include <stdint.h>",
        "static const uint16_t przm_meta8_freq[8][256] = {",
    ]
    for row in rows:
        out.append("  {")
        for i in range(0, 256, 16):
            out.append("    " + ", ".join(str(v) for v in row[i:i + 16]) + ",")
        out.append("  },")
    out += ["};", "#endif", ""]
    sys.stdout.write("\n".join(out))


if __name__ == "__main__":
    main()
