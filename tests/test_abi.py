"""The C ABI: the library loads without a GPU, exports every declared
symbol, and the ctypes mirror matches the C struct layouts (CPU only)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from nonenone_b200 import abi
from nonenone_b200.lib import EXPORTED, LIB_PATH

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "nonenone_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nz_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_what_the_loader_binds():
    assert set(declared_functions()) == set(EXPORTED)


@pytest.mark.skipif(not os.path.exists(LIB_PATH), reason="library not built")
def test_library_exports_every_declared_symbol():
    lib = C.CDLL(LIB_PATH)
    missing = [s for s in declared_functions() if not hasattr(lib, s)]
    assert not missing, missing
    assert lib.nz_abi_version() == 2


def test_struct_layouts_match_c(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(f'''
#include <stdio.h>
#include <stddef.h>
#include "{HEADER}"
int main(void) {{
  printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(nz_fluid_desc), sizeof(nz_flash_options),
         sizeof(nz_flash_out), sizeof(nz_natural_desc), sizeof(nz_report), sizeof(nz_relperm_desc),
         offsetof(nz_fluid_desc, sw_bip_value));
  return 0;
}}''')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    want = [C.sizeof(abi.FluidDesc), C.sizeof(abi.FlashOptions), C.sizeof(abi.FlashOut),
            C.sizeof(abi.NaturalDesc), C.sizeof(abi.Report), C.sizeof(abi.RelpermDesc),
            abi.FluidDesc.sw_bip_value.offset]
    assert got == want


def test_default_options_match_c():
    lib = pytest.importorskip("nonenone_b200.lib").load() if os.path.exists(LIB_PATH) else None
    if lib is None:
        pytest.skip("library not built")
    o = abi.FlashOptions()
    lib.nz_flash_options_default(C.byref(o))
    d = abi.default_flash_options()
    for name, _ in abi.FlashOptions._fields_:
        assert getattr(o, name) == getattr(d, name), name
