"""Regenerates tests/golden/oracle_golden.json: digests of the oracle's
outputs on small seeded inputs.  Before writing, every frame is decoded by
the reference's own C99 decoder (oracle/_ref/libprzm_dec.so, built from the
reference sources by oracle/Makefile) and must give the input back; the
digests then freeze the oracle's behaviour for the CPU test suite.

usage: python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from przm_b200 import workloads as W  # noqa: E402


def sha(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def main() -> None:
    O.build()
    cases = []
    for kind in ("markov", "table", "records", "uniform"):
        for n in (1000, 40000, 65536, 70001, 300000):
            seed = 0x50525A4D + 17 * n + len(kind)
            a = W.gen(kind, seed, n)
            c, o, l = O.tokenize(a)
            p0, p1 = O.compress_p0(a), O.compress_p1(a)
            assert O.ref_decompress(p1, n) == a.tobytes()
            if not O.raw_literals_misparse(l):
                assert O.ref_decompress(p0, n) == a.tobytes()
            vh = O.vans_encode_host(a)
            assert O.ref_decode_vans_literals(vh) == a.tobytes()
            cases.append({
                "name": f"{kind}-{n}", "kind": kind, "seed": seed, "n": n,
                "input_sha256": sha(a.tobytes()),
                "match_table_sha256": sha(O.match_table(a).tobytes()),
                "tokens_sha256": sha(c + b"|" + o + b"|" + l),
                "p0_sha256": sha(p0), "p1_sha256": sha(p1), "vans_host_sha256": sha(vh),
                "p0_size": len(p0), "p1_size": len(p1),
            })
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle_golden.json")
    json.dump({"generator": "tests/golden/make_golden.py", "cases": cases}, open(out, "w"), indent=1)
    print(f"wrote {len(cases)} cases to {out}")


if __name__ == "__main__":
    main()
