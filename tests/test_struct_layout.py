"""The Python mirrors of the C ABI's structs have the C layout (no GPU).

clwilson_b200 passes wl_result, wl_row, wl_range, wl_range_result, wl_stats,
wl_tuning, wl_server_opts, wl_request_info and wl_server_stats across the C
ABI as ctypes structures.  A field added to one side only, or in another
order, would shift every later field and pass garbage without an error.  This
compiles include/wilson.h with the host C compiler and checks each struct's
size and each mirrored field's offset against the ctypes structure.
"""
import ctypes
import os
import shutil
import subprocess

import pytest

import clwilson_b200 as wl

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

MIRRORS = {
    "wl_result": wl._Result,
    "wl_row": wl._Row,
    "wl_range": wl._Range,
    "wl_range_result": wl._RangeResult,
    "wl_stats": wl._Stats,
    "wl_tuning": wl._Tuning,
    "wl_server_opts": wl._ServerOpts,
    "wl_request_info": wl._RequestInfo,
    "wl_server_stats": wl._ServerStats,
}


def _c_layout(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no host C compiler")
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "wilson.h"', "int main(void) {"]
    for cname, py in MIRRORS.items():
        lines.append('    printf("%s sizeof %%zu\\n", sizeof(%s));' % (cname, cname))
        for field, _ in py._fields_:
            lines.append('    printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, field, cname, field))
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.check_call([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    out = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        cname, field, value = line.split()
        out[(cname, field)] = int(value)
    return out


def test_ctypes_mirrors_match_the_header(tmp_path):
    c = _c_layout(tmp_path)
    for cname, py in MIRRORS.items():
        assert ctypes.sizeof(py) == c[(cname, "sizeof")], cname
        for field, _ in py._fields_:
            assert getattr(py, field).offset == c[(cname, field)], (cname, field)
