"""The C ABI's structs as a C compiler lays them out (include/gsn.h, compiled
here with gcc) against their ctypes mirrors in gsn.py: the size of every struct
and the offset of every field, so that an option or a buffer pointer can never
land in the wrong slot."""
import ctypes
import os
import shutil
import subprocess

import pytest

import gsn

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# C struct name -> ctypes mirror
MIRRORS = {
    "gsn_camera": gsn.Camera,
    "gsn_renderer_buffers": gsn.RendererBuffers,
    "gsn_training_options": gsn.TrainingOptions,
}


def _c_layout(tmp_path):
    if shutil.which("gcc") is None:
        pytest.skip("gcc is not installed")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "gsn.h"', "int main(void) {"]
    for cname, mirror in MIRRORS.items():
        lines.append(f'    printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for field, _ in mirror._fields_:
            lines.append(f'    printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True,
                   capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    layout = {}
    for line in out.splitlines():
        cname, key, value = line.split()
        layout[(cname, key)] = int(value)
    return layout


@pytest.mark.parametrize("cname", sorted(MIRRORS))
def test_struct_layout_matches_the_header(cname, tmp_path):
    layout = _c_layout(tmp_path)
    mirror = MIRRORS[cname]
    assert ctypes.sizeof(mirror) == layout[(cname, "sizeof")]
    for field, _ in mirror._fields_:
        assert getattr(mirror, field).offset == layout[(cname, field)], field
