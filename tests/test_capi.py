"""libz80b200.so loads without a GPU and exports every function that
include/z80b200.h declares; the product fails loudly when no device exists."""
import ctypes
import os
import re

import pytest

import z80b
from conftest import ROOT


def declared_functions():
    text = open(os.path.join(ROOT, "include", "z80b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(z80b_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ["z80b_init", "z80b_quickcheck", "z80b_search", "z80b_load_candidates",
              "z80b_fingerprints", "z80b_verify_pairs", "z80b_rules_json"]:
        assert n in names


def test_library_exports_all_declared():
    lib = z80b.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(z80b.EXPORTS) <= set(declared_functions())


def test_status_strings():
    lib = z80b.lib()
    lib.z80b_status_string.restype = ctypes.c_char_p
    assert lib.z80b_status_string(0) == b"ok"
    assert lib.z80b_status_string(5) == b"output buffer too small"


def test_init_without_device_fails_loudly():
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(z80b.Z80BError) as e:
        z80b.Context(0)
    assert e.value.status == z80b.ENODEV


def test_option_numbers_match_header():
    """The Python binding's option constants are the header's Z80B_OPT_*."""
    text = open(os.path.join(ROOT, "include", "z80b200.h")).read()
    defs = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define Z80B_(OPT_\w+)\s+(\d+)", text)}
    assert len(defs) >= 10
    for name, value in defs.items():
        assert getattr(z80b, name) == value, name
