"""The Python mirror's ctypes structures against the C ABI header: every struct
that crosses the boundary has the same size and every field the same offset,
as gcc lays them out from include/vpfft_capi.h.  A field added to the header
but not to the mirror (or the other way round) shifts the offsets and fails
here, before any call could read or write the wrong bytes."""
import ctypes
import os
import shutil
import subprocess

import pytest

from vpfft_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PAIRS = [
    ("vpfft_material", capi.Material),
    ("vpfft_solver_options", capi.SolverOptions),
    ("vpfft_stats", capi.Stats),
    ("vpfft_config", capi.Config),
    ("vpfft_batch_options", capi.BatchOptions),
    ("vpfft_tile_tuning", capi.TileTuning),
    ("vpfft_batch_result", capi.BatchResult),
    ("vpfft_batch_info", capi.BatchInfo),
]


def c_layout(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "vpfft_capi.h"',
             'int main(void) {']
    for cname, py in PAIRS:
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, *_ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ['  return 0;', '}']
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                    str(exe)], check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    table = {}
    for line in out.splitlines():
        name, field, value = line.split()
        table[(name, field)] = int(value)
    return table


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_structs_match_the_c_header(tmp_path):
    table = c_layout(tmp_path)
    for cname, py in PAIRS:
        assert table[(cname, "size")] == ctypes.sizeof(py), cname
        for fname, *_ in py._fields_:
            assert table[(cname, fname)] == getattr(py, fname).offset, (cname, fname)
