"""Regenerates the golden fixtures of tests/golden/ (run in a checkout that has
the reference sources; nothing in the test suite reads the reference itself).

partitions_ref.json
    Basis rows produced by the reference's own generator
    (modules/partitions/integer_partitions.cu), compiled from its sources by
    ``make -C oracle ref`` into oracle/_ref/ref_partitions and run on the CPU.
philox_kat.json
    Known-answer vectors of Philox-4x32-10 published with Random123
    (Salmon et al., SC'11, kat_vectors), restated as numbers.
"""
import hashlib
import json
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
REF_BIN = ROOT / "oracle" / "_ref" / "ref_partitions"

CASES = [
    (8, list(range(0, 7))),       # plain method, small size (dL = 1..6 plus the ground state)
    (3, [4, 5, 6]),               # more parts than particles: the <= N filter
    (50, list(range(0, 13))),     # mixed-precision form
    (100, [16, 20]),
    (200, [0, 1, 2]),
]
HASH_CASES = [(100, list(range(1, 21)))]  # batched form: 2713 rows, stored as counts + sha256


def run_ref(N, sectors):
    out = subprocess.run([str(REF_BIN), str(N)] + [str(s) for s in sectors], capture_output=True,
                         text=True, check=True).stdout
    rows, meta = [], None
    for line in out.splitlines():
        if line.startswith("META"):
            meta = [int(x) for x in line.split()[1:]]
        elif line.startswith("ROW"):
            f = line.split()
            pairs = [[int(a) for a in t.split("x")] for t in f[3:]]
            rows.append({"dL": int(f[1]), "sector_size": int(f[2]), "pairs": pairs})
    return meta, rows


def canonical(rows):
    return "\n".join(f"{r['dL']} " + " ".join(f"{p}x{m}" for p, m in r["pairs"]) for r in rows)


def main():
    if not REF_BIN.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "ref"], check=True)
    cases = []
    for N, secs in CASES:
        meta, rows = run_ref(N, secs)
        cases.append({"N": N, "sectors": secs, "dim": meta[0], "max_degree": meta[1],
                      "longest": meta[2], "rows": rows})
    hashed = []
    for N, secs in HASH_CASES:
        meta, rows = run_ref(N, secs)
        counts = [sum(1 for r in rows if r["dL"] == s) for s in secs]
        hashed.append({"N": N, "sectors": secs, "dim": meta[0], "max_degree": meta[1],
                       "longest": meta[2], "counts": counts,
                       "sha256": hashlib.sha256(canonical(rows).encode()).hexdigest()})
    (HERE / "partitions_ref.json").write_text(json.dumps({"source": "reference integer_partitions.cu",
                                                         "cases": cases, "hashed": hashed}))
    kat = {"source": "Random123 kat_vectors, philox4x32 R=10",
           "vectors": [
               {"ctr": [0, 0, 0, 0], "key": [0, 0],
                "out": [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]},
               {"ctr": [0xffffffff] * 4, "key": [0xffffffff] * 2,
                "out": [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]},
               {"ctr": [0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344],
                "key": [0xa4093822, 0x299f31d0],
                "out": [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]}]}
    (HERE / "philox_kat.json").write_text(json.dumps(kat, indent=1))


if __name__ == "__main__":
    main()
