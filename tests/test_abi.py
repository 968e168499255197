"""The C-ABI library loads and exports every entry point include/tapsim_gpu.h declares."""
import re
import subprocess
from pathlib import Path

from conftest import ROOT

HEADER = ROOT / "include" / "tapsim_gpu.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tg_\w+)\s*\(", text)))


def test_library_loads_and_exports_header_symbols():
    from tapsim_modified_b200 import _native as N
    L = N.lib()
    names = declared_functions()
    assert len(names) >= 30
    for name in names:
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(N.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (tg_\w+)", out))
    assert set(names) <= exported


def test_ctypes_signatures_cover_header():
    from tapsim_modified_b200 import _native as N
    assert set(N.SIGNATURES) == set(declared_functions())


def test_struct_sizes_match_c_layout():
    """ctypes mirrors of the ABI structs have the C sizes (compiled probe)."""
    import ctypes as C
    from tapsim_modified_b200 import _native as N
    probe = ROOT / "tapsim_modified_b200" / "_build" / "abi_sizes"
    src = probe.with_suffix(".c")
    src.parent.mkdir(exist_ok=True)
    src.write_text('#include <stdio.h>\n#include "tapsim_gpu.h"\nint main(){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu\\n",'
                   "sizeof(tg_type),sizeof(tg_mesh_desc),sizeof(tg_solve_opts),sizeof(tg_solve_info),"
                   "sizeof(tg_select_info),sizeof(tg_trace_opts),sizeof(tg_impact),sizeof(tg_event_opts),"
                   "sizeof(tg_event_record));return 0;}\n")
    subprocess.run(["gcc", "-I", str(ROOT / "include"), "-o", str(probe), str(src)], check=True)
    sizes = list(map(int, subprocess.run([str(probe)], capture_output=True, text=True).stdout.split()))
    mirrors = [N.tg_type, N.tg_mesh_desc, N.tg_solve_opts, N.tg_solve_info, N.tg_select_info, N.tg_trace_opts,
               N.tg_impact, N.tg_event_opts, N.tg_event_record]
    assert sizes == [C.sizeof(m) for m in mirrors]


def test_device_entry_points_fail_cleanly_without_gpu():
    """Without a device, tg_create reports TG_ERR_CUDA instead of crashing."""
    import ctypes as C
    import pytest
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    from tapsim_modified_b200 import _native as N
    d = N.tg_mesh_desc()
    h = C.c_void_p()
    assert N.lib().tg_create(C.byref(d), C.byref(h)) == 1   # incomplete description: argument error
