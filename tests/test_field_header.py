"""include/psr_field.cuh compiles into an application's own kernels (no GPU needed): the
user kernel of the device-field GPU test builds with nvcc's default flags through
warp_psr_b200.build.build_user_library, and the handle layout matches its ctypes mirror."""
import ctypes
import re
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(not (shutil.which("nvcc") or Path("/usr/local/cuda/bin/nvcc").exists()), reason="no nvcc")
def test_user_kernel_builds_against_the_header(tmp_path):
    from warp_psr_b200.build import build_user_library
    out = build_user_library([ROOT / "tests" / "kernels" / "device_field_user.cu"], tmp_path / "libuser.so")
    text = out.read_bytes()
    assert b"user_evaluate" in text


def test_handle_mirror_matches_the_header():
    from warp_psr_b200 import _lib
    header = (ROOT / "include" / "psr_b200.h").read_text()
    body = re.search(r"typedef struct psr_field_handle \{(.*?)\} psr_field_handle;", header, re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    names = re.findall(r"(\w+)(?:\[\d+\])?;", body)
    assert names == [f[0] for f in _lib.FieldHandle._fields_]


@pytest.mark.skipif(not shutil.which("gcc"), reason="no C compiler")
def test_handle_offsets_match_the_c_layout(tmp_path):
    from warp_psr_b200 import _lib
    fields = [f[0] for f in _lib.FieldHandle._fields_]
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "psr_b200.h"\nint main(void) {\n'
                   + "".join(f'  printf("%zu\\n", offsetof(psr_field_handle, {f}));\n' for f in fields)
                   + '  printf("%zu\\n", sizeof(psr_field_handle));\n  return 0;\n}\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got[:-1] == [getattr(_lib.FieldHandle, f).offset for f in fields]
    assert got[-1] == ctypes.sizeof(_lib.FieldHandle)
