"""The C ABI library loads and matches include/pscf_gpu.h (no GPU needed)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from pscf_b200 import engine as E

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pscf_gpu.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pscfg_[a-z_0-9]+)\s*\(", text)))


def test_header_functions_exported_and_bound():
    lib = E.load_library()
    decl = declared_functions()
    assert len(decl) >= 15
    for name in decl:
        assert hasattr(lib, name), name          # exported by libpscfgpu.so
        assert name in E.SIGNATURES, name        # bound by the Python layer
    assert set(E.SIGNATURES) == set(decl)


def test_library_has_no_oracle_dependency():
    out = subprocess.run(["nm", "-D", "--defined-only", E.LIB_PATH], capture_output=True, text=True).stdout
    assert "orc_" not in out
    deps = subprocess.run(["ldd", E.LIB_PATH], capture_output=True, text=True).stdout
    assert "oracle" not in deps


@pytest.mark.parametrize("struct,cname", [(E.PscfgSystem, "pscfg_system"), (E.PscfgAmParam, "pscfg_am_param"),
                                          (E.PscfgAmResult, "pscfg_am_result")])
def test_struct_layout_matches_header(struct, cname):
    fields = [f[0] for f in struct._fields_]
    body = "\n".join('printf("%s %%zu\\n", offsetof(%s, %s));' % (f, cname, f) for f in fields)
    src = '#include <stdio.h>\n#include <stddef.h>\n#include "pscf_gpu.h"\nint main(void){printf("size %%zu\\n", sizeof(%s));%s return 0;}\n' % (cname, body)
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "p.c")
        exe = os.path.join(d, "p")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    vals = dict(line.split() for line in out if line)
    assert int(vals["size"]) == C.sizeof(struct)
    for f in fields:
        assert int(vals[f]) == getattr(struct, f).offset, f


def test_create_rejects_bad_input_without_gpu_work():
    """Argument validation happens before any device call."""
    lib = E.load_library()
    h = C.c_void_p()
    assert lib.pscfg_create(None, 1, 0, C.byref(h)) == E.EINVAL
    assert b"null" in lib.pscfg_last_error(None)
