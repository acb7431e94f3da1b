"""The Python binding's ctypes mirrors of the C-ABI structs have the C
layout: every field at the offset that include/silvan.h gives it, and the
same struct size.  A C program built here with gcc prints sizeof and offsetof
for every field the binding names (no GPU needed)."""
import os
import subprocess

import pytest

from conftest import ROOT

# binding class -> (C typedef, {binding field: C field})
STRUCTS = {
    "GraphInfo": ("silvan_graph_info_t", {}),
    "Params": ("silvan_params_t", {}),
    "Result": ("silvan_result_t", {}),
    "Status": ("silvan_status_t", {"pass_": "pass"}),
    "ServerStats": ("silvan_server_stats_t", {}),
}


@pytest.fixture(scope="module")
def c_layout(sb, tmp_path_factory):
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "silvan.h"', "int main(void) {"]
    for cls, (ctype, rename) in STRUCTS.items():
        lines.append(f'    printf("{cls} size %zu\\n", sizeof({ctype}));')
        for f, _ in getattr(sb, cls)._fields_:
            cf = rename.get(f, f)
            lines.append(f'    printf("{cls} {f} %zu\\n", offsetof({ctype}, {cf}));')
    lines += ["    return 0;", "}"]
    d = tmp_path_factory.mktemp("abi")
    src, exe = d / "layout.c", d / "layout"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                    str(exe)], check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    layout = {}
    for line in out.splitlines():
        cls, field, value = line.split()
        layout[(cls, field)] = int(value)
    return layout


@pytest.mark.parametrize("cls", sorted(STRUCTS))
def test_binding_struct_matches_header(sb, c_layout, cls):
    import ctypes
    py = getattr(sb, cls)
    assert ctypes.sizeof(py) == c_layout[(cls, "size")]
    for f, _ in py._fields_:
        assert getattr(py, f).offset == c_layout[(cls, f)], (cls, f)
