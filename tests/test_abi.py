"""The C-ABI library loads and exports every symbol include/*.h declares (no GPU calls)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

from scout_b200 import _lib

DECL = re.compile(r"^(?:int|int64_t|void|const char\s*\*|const int32_t\s*\*|const int64_t\s*\*|scout_ctx\s*\*)"
                  r"\s*\*?\s*(scout_\w+)\s*\(", re.M)


def _declared():
    names = set()
    for h in ("scout_gpu.h", "scout_host.h"):
        names |= set(DECL.findall(open(os.path.join(ROOT, "include", h)).read()))
    return names


def test_every_declared_symbol_is_exported():
    names = _declared()
    assert len(names) > 50
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_signatures_cover_the_headers():
    bound = {n for n, _, _ in _lib.SIGNATURES}
    assert _declared() - bound == set()


def test_no_device_path_fails_cleanly():
    import scout_b200 as sb
    if sb.device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(sb.ScoutError) as e:
        sb.Context(0)
    assert e.value.code == -8   # SCOUT_E_NODEV, no crash, no exit
