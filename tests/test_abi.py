"""CPU tests of the C-ABI boundary: the library loads and exports every declared symbol (no GPU calls)."""
import ctypes
import re
from pathlib import Path

from tensorjoin_variants_b200 import _lib

HEADER = Path(__file__).resolve().parents[1] / "include" / "tensorjoin.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(tj_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_expected_api():
    assert set(declared_functions()) == set(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    for name in declared_functions():
        assert hasattr(L, name), name
    assert L.tj_version() == 1
    assert isinstance(L.tj_last_error_string(), (bytes, type(None)))


def test_structs_match_header_layout():
    assert ctypes.sizeof(_lib.Options) == 24
    assert ctypes.sizeof(_lib.Stats) == 11 * 8 + 9 * 8 + 8 + 8 + 8 + 8 + 8 + 4 * 8 + 9 * 8
    assert ctypes.sizeof(_lib.BatchJoin) == 48


def test_flag_constants_match_header():
    text = HEADER.read_text()
    flags = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define TJ_FLAG_([A-Z0-9_]+) (\d+)", text)}
    assert flags, "no TJ_FLAG_* defines found"
    for name, value in flags.items():
        assert getattr(_lib, "FLAG_" + name) == value, name
    assert len(set(flags.values())) == len(flags)


def _header_struct(name):
    """(field, C type) pairs of `typedef struct name { ... } name;` in declaration order."""
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), text, flags=re.S).group(1)
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        m = re.match(r"((?:const )?[a-z0-9_]+\*?)\s+(.*)", decl)
        ctype, names = m.group(1), m.group(2)
        for nm in names.split(","):
            fields.append((nm.strip().lstrip("*"), ctype))
    return fields


CTYPES = {"int64_t": ctypes.c_int64, "int32_t": ctypes.c_int32, "double": ctypes.c_double,
          "const void*": ctypes.c_void_p}


def test_structs_match_header_fields():
    """Every ctypes mirror lists the header's fields in the header's order with the same types."""
    for cname, pystruct in (("tj_options", _lib.Options), ("tj_stats", _lib.Stats),
                            ("tj_batch_join", _lib.BatchJoin)):
        hdr = _header_struct(cname)
        py = [(n, t) for n, t in pystruct._fields_]
        assert [n for n, _ in hdr] == [n for n, _ in py], cname
        for (n, ht), (_, pt) in zip(hdr, py):
            assert CTYPES[ht] is pt, (cname, n, ht, pt)
