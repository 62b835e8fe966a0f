"""lemc_partitions (the library's basis enumeration) against the reference generator."""
import hashlib
import json
from pathlib import Path

GOLD = Path(__file__).resolve().parent / "golden"


def _canon(rows):
    return "\n".join(f"{dl} " + " ".join(f"{p}x{m}" for p, m in pr) for dl, pr in rows)


def test_library_partitions_match_reference(lemc):
    gold = json.loads((GOLD / "partitions_ref.json").read_text())
    for case in gold["cases"]:
        rows, maxdeg, longest = lemc.partitions(case["N"], case["sectors"])
        assert len(rows) == case["dim"]
        assert maxdeg == case["max_degree"]
        assert longest == case["longest"]
        for got, want in zip(rows, case["rows"]):
            assert got[0] == want["dL"]
            assert [list(p) for p in got[1]] == want["pairs"]
    for case in gold["hashed"]:
        rows, maxdeg, longest = lemc.partitions(case["N"], case["sectors"])
        assert len(rows) == case["dim"] and maxdeg == case["max_degree"]
        assert longest == case["longest"]
        assert [sum(1 for r in rows if r[0] == s) for s in case["sectors"]] == case["counts"]
        assert hashlib.sha256(_canon(rows).encode()).hexdigest() == case["sha256"]


def test_partitions_bad_arguments(lemc):
    import ctypes as C
    import numpy as np
    lib = lemc.load()
    sec = np.array([3], np.int32)
    n = C.c_int()

    assert lib.lemc_partitions(0, lemc._lib.i32ptr(sec), 1, None, 0, None, 0, C.byref(n), None,
                               None, None) == -1
    neg = np.array([-1], np.int32)
    assert lib.lemc_partitions(4, lemc._lib.i32ptr(neg), 1, None, 0, None, 0, C.byref(n), None,
                               None, None) == -1
