"""The Python bindings' ctypes mirrors of the C-ABI structs have the header's layout: a
small C program built with gcc against include/cavalry.h prints each struct's size and
every field's offset, and the ctypes classes must agree (no GPU needed)."""
import ctypes
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent

PAIRS = {  # C struct -> ctypes class name in cavalry_b200
    "cav_scene_info_t": "SceneInfo",
    "cav_render_opts": "RenderOpts",
    "cav_render_stats_t": "RenderStats",
    "cav_guide_opts": "GuideOpts",
    "cav_guide_stats": "GuideStats",
    "cav_server_config": "ServerConfig",
    "cav_job_status": "JobStatus",
    "cav_server_stats_t": "ServerStats",
    "cav_trace_config_t": "TraceConfig",
    "cav_scene_job": "SceneJob",
}


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    import cavalry_b200 as cav

    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "cavalry.h"', "int main(void) {"]
    for c_name, py_name in PAIRS.items():
        cls = getattr(cav, py_name)
        lines.append(f'  printf("{c_name} size %zu\\n", sizeof({c_name}));')
        for field, _ in cls._fields_:
            lines.append(f'  printf("{c_name} {field} %zu\\n", offsetof({c_name}, {field}));')
    lines += ["  return 0;", "}"]
    d = tmp_path_factory.mktemp("abi")
    src, exe = d / "layout.c", d / "layout"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run(["gcc", "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True,
                   capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    table = {}
    for line in out.splitlines():
        s, f, v = line.split()
        table[(s, f)] = int(v)
    return table


@pytest.mark.parametrize("c_name", list(PAIRS))
def test_ctypes_mirror_matches_header(c_layout, c_name):
    import cavalry_b200 as cav

    cls = getattr(cav, PAIRS[c_name])
    assert ctypes.sizeof(cls) == c_layout[(c_name, "size")], c_name
    for field, _ in cls._fields_:
        assert getattr(cls, field).offset == c_layout[(c_name, field)], (c_name, field)
