"""The C ABI: header <-> Python mirror agreement, and the library exports every declared symbol.

No compute calls here (these run without a GPU)."""
import ctypes
import os
import re
import subprocess

import pytest

from polymer_dns_b200 import abi, runtime

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "kmm.h")


def _header():
    with open(HEADER) as f:
        return f.read()


def _strip_comments(s):
    s = re.sub(r"/\*.*?\*/", "", s, flags=re.S)
    return re.sub(r"//[^\n]*", "", s)


def test_param_struct_matches_header():
    h = _strip_comments(_header())
    body = re.search(r"typedef struct kmm_params \{(.*?)\} kmm_params;", h, re.S).group(1)
    members = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        typ, names = decl.split(None, 1)
        for n in names.split(","):
            members.append((n.strip(), typ))
    py = [(n, "double" if t is ctypes.c_double else "int") for n, t in abi.KmmParams._fields_]
    assert members == py


def test_field_ids_match_header():
    h = _strip_comments(_header())
    body = re.search(r"enum kmm_field \{(.*?)\};", h, re.S).group(1)
    val = -1
    ids = {}
    for tok in body.replace("\n", " ").split(","):
        tok = tok.strip()
        if not tok:
            continue
        if "=" in tok:
            name, v = [t.strip() for t in tok.split("=")]
            val = int(v)
        else:
            name = tok
            val += 1
        ids[name] = val
    for name, v in ids.items():
        key = name[len("KMM_"):]
        if key.endswith("_END"):
            continue
        assert abi.FIELD[key] == v, name


def test_status_codes_match_header():
    h = _strip_comments(_header())
    body = re.search(r"enum kmm_status \{(.*?)\};", h, re.S).group(1)
    for m in re.finditer(r"(KMM_\w+)\s*=\s*(\d+)", body):
        assert abi.STATUS_NAMES[int(m.group(2))] == m.group(1)


def test_header_declares_every_python_routine():
    h = _header()
    for sym in runtime.exported_symbols():
        assert re.search(r"\b%s\s*\(" % sym, h), sym


def test_library_exports_every_header_symbol():
    from polymer_dns_b200 import build
    lib = build.build()
    out = subprocess.check_output(["nm", "-D", "--defined-only", lib]).decode()
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    declared = set(re.findall(r"\b(kmm_\w+)\s*\(", _strip_comments(_header())))
    missing = sorted(declared - exported)
    assert not missing, missing
    # and it loads (no compute call without a GPU)
    L = runtime.lib()
    assert L.kmm_abi_version() == abi.KMM_ABI_VERSION
