"""The C-ABI library loads and exports every symbol include/lemc.h declares."""
import ctypes as C
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _declared():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        names |= set(re.findall(r"^LEMC_API\s+[\w\s\*]+?\b(lemc_\w+)\s*\(", h.read_text(), re.M))
    return names


def test_every_declared_symbol_is_exported(lemc):
    names = _declared()
    assert len(names) >= 20
    lib = C.CDLL(str(lemc._lib.LIB_PATH))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_declarations(lemc):
    assert _declared() <= set(lemc._lib._SIGNATURES)


def test_status_strings_and_version(lemc):
    lib = lemc.load()
    assert lib.lemc_version() >= 10000
    for s in (0, -1, -2, -4, -5, -6, -7, -8):
        assert lib.lemc_status_string(s)


def test_create_rejects_bad_config_without_touching_the_device(lemc):
    lib = lemc.load()
    h = C.c_void_p()
    cfg = lemc._lib.Config(1, 3, 16, 0, 0.3, 0, 42, 0.0, 0.0, 0, 0, 0, 0)  # one particle
    assert lib.lemc_create(C.byref(cfg), C.byref(h)) == -1
    cfg = lemc._lib.Config(8, 3, 16, 0, -1.0, 0, 42, 0.0, 0.0, 0, 0, 0, 0)  # bad step
    assert lib.lemc_create(C.byref(cfg), C.byref(h)) == -1
    assert lib.lemc_create(None, C.byref(h)) == -1
