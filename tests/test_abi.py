"""libpbrcm.so loads without a GPU and exports exactly what include/pbrcm.h
declares, with the struct layouts the header defines."""
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "pbrcm.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"PBRCM_API\s+[\w\s\*]+?\b(pbrcm_\w+)\s*\(", text)))


def test_header_declares_functions():
    assert len(declared_functions()) >= 20


def test_library_exports_every_declared_symbol(pbrcm):
    from parallelbatchrcm_b200 import _lib
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.lib_path()], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (pbrcm_\w+)", out))
    missing = [f for f in declared_functions() if f not in exported]
    assert not missing, missing
    # and the Python binding knows every one of them
    assert set(declared_functions()) == set(_lib.SIGNATURES)


def test_checks_build_exports_the_same(pbrcm):
    from parallelbatchrcm_b200 import _lib
    if not os.path.exists(_lib.CHECKS_LIB):
        pytest.skip("checks build not present")
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.CHECKS_LIB], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (pbrcm_\w+)", out))
    assert set(declared_functions()) <= exported


def test_struct_layouts_match_header(tmp_path):
    """Compiles the header with the host C compiler and compares sizeof /
    offsetof with the ctypes mirrors."""
    import ctypes
    from parallelbatchrcm_b200 import _lib
    structs = {"pbrcm_options": _lib.Options, "pbrcm_result": _lib.Result, "pbrcm_matrix": _lib.Matrix,
               "pbrcm_session_config": _lib.SessionConfig, "pbrcm_session_stats": _lib.SessionStats}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', 'int main(void){']
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-o", str(exe), str(src)], check=True)
    got = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                               check=True).stdout.splitlines())
    for cname, py in structs.items():
        assert int(got[cname]) == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(py, fname).offset, (cname, fname)


def test_status_strings(pbrcm):
    from parallelbatchrcm_b200 import _lib
    L = _lib.lib()
    assert L.pbrcm_status_string(0) == b"ok"
    assert b"connected" in L.pbrcm_status_string(2)
    assert L.pbrcm_version().startswith(b"pbrcm-b200")


def test_prepared_batch_descriptors():
    """The binding's batch descriptors (pbrcm_matrix) carry each buffer's
    address and sizes; results come back as a sequence of dicts."""
    import numpy as np
    from parallelbatchrcm_b200 import rcm
    from parallelbatchrcm_b200._lib import Result
    mats = [(np.array([0, 1, 2], dtype=np.uint32), np.array([1, 0], dtype=np.uint32)),
            (np.array([0, 0], dtype=np.uint32), np.zeros(0, dtype=np.uint32))]
    pb = rcm.PreparedBatch(mats)
    assert pb.count == 2 and not pb.device
    for i, (rp, ci) in enumerate(pb.mats):
        d = pb.arr[i]
        assert d.row_ptr == rp.ctypes.data and (d.col_idx or 0) == ci.ctypes.data
        assert d.n == rp.shape[0] - 1 and d.nnz == ci.shape[0]
        assert d.perm_out == pb.perms[i].ctypes.data
    res = (Result * 3)()
    res[2].status = 9
    br = rcm.BatchResults(res)
    assert len(br) == 3 and br[-1]["status"] == 9 and [r["status"] for r in br] == [0, 0, 9]
