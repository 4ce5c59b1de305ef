"""The C-ABI library loads without a GPU and exports every entry point declared in include/edipic_gpu.h, and
the ctypes mirrors have the C structure sizes."""
import ctypes as C
import os
import re
import shutil
import subprocess

import pytest

from edipic_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "edipic_gpu.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*int\s+(edp_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = _abi.load()
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(_abi.SIGNATURES), "ctypes signature table out of date"


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_struct_sizes_match_header(tmp_path):
    prog = tmp_path / "sz.c"
    prog.write_text('#include "edipic_gpu.h"\n#include <stdio.h>\n#include <stddef.h>\n'
                    'int main(){printf("%zu %zu %zu %zu %zu\\n", sizeof(edp_params), sizeof(edp_tables),'
                    ' sizeof(edp_counters), offsetof(edp_params, seed), offsetof(edp_tables, maxwell_v));return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(prog), "-o", str(exe)])
    sizes = [int(x) for x in subprocess.check_output([str(exe)]).split()]
    assert sizes == [C.sizeof(_abi.Params), C.sizeof(_abi.Tables), C.sizeof(_abi.Counters),
                     _abi.Params.seed.offset, _abi.Tables.maxwell_v.offset]


def test_init_rejects_bad_arguments_without_gpu():
    lib = _abi.load()
    p = _abi.Params()
    t = _abi.Tables()
    ctx = C.c_void_p()
    assert lib.edp_init(C.byref(p), C.byref(t), C.byref(ctx)) == _abi.ERR_ARG   # wrong ABI version
    assert lib.edp_destroy(None) == 0


def test_init_limits_without_gpu(tmp_path):
    """edp_init checks its arguments before it looks for a device: an FFT_X grid beyond 4096 columns or not a power
    of two, a negative permittivity, and a dielectric object with the FFT_X solver are refused."""
    from edipic_b200 import decks, read_deck
    d = read_deck(decks.write_deck(str(tmp_path), "cfg0", ncx=64, ncy=32, ppc=4))
    lib = _abi.load()
    ctx = C.c_void_p()
    p = _abi.Params.from_buffer_copy(d.params)
    assert lib.edp_init(C.byref(p), C.byref(d.tables), C.byref(ctx)) == _abi.ERR_CUDA   # valid: fails on no device
    for change in ({"ncx": 8192}, {"ncx": 96}, {"n_inner": 1, "eps": -1.0}, {"n_inner": 1, "eps": 2.0}):
        p = _abi.Params.from_buffer_copy(d.params)
        if "ncx" in change:
            p.ncx = change["ncx"]
        if "n_inner" in change:
            p.n_inner = 1
            p.inner_ileft[0], p.inner_jbottom[0], p.inner_iright[0], p.inner_jtop[0] = 10, 10, 20, 20
            p.inner_eps[0] = change["eps"]
        assert lib.edp_init(C.byref(p), C.byref(d.tables), C.byref(ctx)) == _abi.ERR_ARG, change
