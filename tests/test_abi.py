"""The C ABI library loads and exports every entry point include/csm_gpu.h
declares (no GPU needed: nothing here calls into the device)."""
from __future__ import annotations

import ctypes
import re
import subprocess
from pathlib import Path

from paracosm_b200 import _abi

HEADER = Path(__file__).resolve().parents[1] / "include" / "csm_gpu.h"


def declared_symbols() -> set[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(csm_gpu_\w+)\s*\(", text))


def test_header_declares_the_python_binding_list():
    assert declared_symbols() == set(_abi.EXPORTED)


def test_library_loads_and_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(_abi.LIB_PATH))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_struct_layouts_match_the_header(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include "csm_gpu.h"\n#include <stdio.h>\n#include <stddef.h>\n'
                   'int main(void){printf("%zu %zu %zu %zu %zu\\n", sizeof(csm_cfg), sizeof(csm_update),'
                   ' sizeof(csm_result), sizeof(csm_stats), offsetof(csm_cfg, vertex_headroom));'
                   'printf("%zu\\n", sizeof(csm_index_info));return 0;}')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", str(HEADER.parent), str(src), "-o", str(exe)], check=True)
    cfg, upd, res, stats, off, info = map(int, subprocess.run([str(exe)], capture_output=True, text=True).stdout.split())
    assert cfg == ctypes.sizeof(_abi.CsmCfg)
    assert off == _abi.CsmCfg.vertex_headroom.offset
    assert upd == _abi.UPDATE_DTYPE.itemsize == 16
    assert res == _abi.RESULT_DTYPE.itemsize == 48
    assert stats == ctypes.sizeof(_abi.CsmStats)
    assert info == ctypes.sizeof(_abi.CsmIndexInfo)


def test_error_strings_without_a_device():
    lib = _abi.load_library()
    assert lib.csm_gpu_strerror(_abi.CSM_EINVAL) == b"invalid argument"
    cfg = _abi.CsmCfg()
    lib.csm_gpu_default_cfg(ctypes.byref(cfg))
    assert cfg.max_batch == 65536 and cfg.mode == _abi.MODE_BATCHED
