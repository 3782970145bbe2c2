"""The ctypes mirrors of the C ABI's structs (pennant_b200 Python binding)
have the C compiler's layout: the same size and, for every field, the same
offset as gcc gives the declarations in include/pennant_b200.h."""
import ctypes as C
import os
import subprocess

import pytest

from conftest import ROOT
import pennant_b200 as pb

STRUCTS = {"pnt_params": pb.Params, "pnt_scalars": pb.Scalars, "pnt_mesh_desc": pb.MeshDesc,
           "pnt_piece_desc": pb.PieceDesc, "pnt_piece_buffers": pb.PieceBuffers}


def _c_layout(tmp_path):
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "pennant_b200.h"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'    printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'    printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                    str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    return {tuple(line.split()[:2]): int(line.split()[2]) for line in out.splitlines()}


@pytest.mark.parametrize("cname", sorted(STRUCTS))
def test_ctypes_structs_match_the_c_layout(cname, tmp_path):
    layout = _c_layout(tmp_path)
    py = STRUCTS[cname]
    assert C.sizeof(py) == layout[(cname, "size")], cname
    for fname, _ in py._fields_:
        assert getattr(py, fname).offset == layout[(cname, fname)], (cname, fname)
