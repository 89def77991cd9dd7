"""The C-ABI library loads and exports every entry point the header declares (no GPU work)."""
import ctypes
import os
import re

import numpy as np

from parallel_admm_b200 import backend as B
from parallel_admm_b200 import scene

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_symbols():
    txt = open(os.path.join(ROOT, "include", "admm_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(admm_(?:b200|gnn|learn)_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(B.LIB_PATH)
    declared = _header_symbols()
    assert len(declared) >= 25
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing
    assert sorted(B.exported_symbols()) == declared


def test_errstr_and_abi_rejects_bad_description():
    L = B.lib()
    assert L.admm_b200_errstr(0) == b"ok"
    assert b"overflow" in L.admm_b200_errstr(B.ERR_CONTACT_OVERFLOW)
    assert L.admm_b200_errstr(-99) == b"unknown status"
    # a wrong ABI version is rejected before any device work
    holder = B.DescHolder(scene.cloth_on_box(4))
    holder.desc.abi_version = 999
    h = ctypes.c_void_p()
    rc = L.admm_b200_create(ctypes.byref(holder.desc), 0, ctypes.byref(h))
    assert rc == B.ERR_INVALID and not h.value
    # null arguments
    assert L.admm_b200_step(None, 1, None) == B.ERR_INVALID
    assert L.admm_b200_get_state(None, None, None, 0) == B.ERR_INVALID


def test_desc_struct_layout_matches_header():
    """Field order of the ctypes mirror equals the C struct's (parsed from the header)."""
    txt = open(os.path.join(ROOT, "include", "admm_b200.h")).read()
    body = txt[txt.index("typedef struct AdmmB200Desc {"):txt.index("} AdmmB200Desc;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    names = []
    for line in body.splitlines()[1:]:
        line = line.strip().rstrip(";")
        if not line:
            continue
        decl = line.split(None, 1)[1] if line.startswith(("int32_t", "float", "const")) else line
        decl = decl.replace("const float*", "").replace("const int32_t*", "").replace("float", "")
        decl = decl.replace("int32_t", "").replace("*", "")
        names += [n.strip() for n in decl.split(",") if n.strip()]
    assert names == [f[0] for f in B.AdmmB200Desc._fields_]
