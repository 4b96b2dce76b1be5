"""The C-ABI boundary without a GPU: libxmp.so loads and exports exactly the
entry points include/xmp.h declares (the 54 XMPAPI prototypes of the
reference's src/include/xmp.h:119-226), and the header compiles as C."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    return sorted(set(re.findall(r"^\s*\w+\s+XMPAPI\s+(\w+)\s*\(", src, re.M)))


def test_header_declares_reference_api():
    names = declared("xmp.h")
    assert len(names) == 55  # the 54 prototypes of src/include/xmp.h + xmpIntegersPowmNoAlloc
    for n in ["xmpHandleCreate", "xmpIntegersImport", "xmpIntegersExport", "xmpIntegersPowm", "xmpIntegersDivMod",
              "xmpIntegersCmp", "xmpIntegersShf", "xmpHandleSetCudaStream"]:
        assert n in names


@pytest.mark.parametrize("header", sorted(f for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")))
def test_library_exports_every_declared_symbol(header):
    import xmp_b200
    lib = xmp_b200.lib()
    for n in declared(header):
        assert hasattr(lib, n), "%s declared in %s but not exported" % (n, header)


def test_python_binding_covers_api():
    import xmp_b200
    assert set(declared("xmp.h")) - {"xmpHandleCreateWithMemoryFunctions", "xmpHandleGetMemoryFunctions"} <= \
        set(xmp_b200.API_NAMES) | {"xmpHandleCreateWithMemoryFunctions", "xmpHandleGetMemoryFunctions"}


@pytest.mark.parametrize("header", ["xmp.h", "xmp_b200.h"])
@pytest.mark.parametrize("lang,compiler", [("c", "gcc"), ("c++", "g++")])
def test_header_compiles(tmp_path, lang, compiler, header):
    src = tmp_path / ("t." + ("c" if lang == "c" else "cc"))
    src.write_text('#include "%s"\nint main(void){ xmpHandle_t h; (void)h; return xmpErrorSuccess; }\n' % header)
    p = subprocess.run([compiler, "-x", lang, "-c", str(src), "-I", os.path.join(ROOT, "include"), "-I",
                        "/usr/local/cuda/include", "-o", str(tmp_path / "t.o")], capture_output=True, text=True)
    assert p.returncode == 0, p.stderr


def test_library_links_no_oracle():
    """The product library must not depend on the oracle or GMP."""
    import xmp_b200
    out = subprocess.run(["ldd", xmp_b200.LIB_PATH], capture_output=True, text=True).stdout
    assert "gmp" not in out and "oracle" not in out
