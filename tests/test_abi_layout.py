"""The ctypes mirrors of the C-ABI structs have the header's layout.

A C program built from ``include/steam_b200.h`` with the host's C compiler
prints sizeof and every field's offset of each struct the Python side
passes by pointer or value; the ctypes classes in ``steam_b200._lib`` must
agree field for field (a mismatch would hand the library shifted pointers).
"""

import ctypes
import shutil
import subprocess
from pathlib import Path

import pytest

from steam_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]

# (C type, ctypes class, [(C field, ctypes field)])
STRUCTS = [
    ("steam_region_t", _lib.Region,
     [("shape", "shape"), ("origin", "origin"), ("world", "world"), ("sparsity", "sparsity"),
      ("key", "key")]),
    ("steam_window_t", _lib.Window, [("x0", "x0"), ("x1", "x1"), ("y0", "y0"), ("y1", "y1")]),
    ("steam_sepconv_t", _lib.SepConv,
     [("kz", "kz"), ("ky", "ky"), ("kx", "kx"), ("cz", "cz"), ("cy", "cy"), ("cx", "cx"),
      ("n_z", "n_z"), ("n_y", "n_y"), ("n_x", "n_x"), ("n_pairs", "n_pairs"),
      ("pair_z", "pair_z"), ("pair_y", "pair_y"), ("mix", "mix")]),
    ("steam_conv_problem_t", _lib.ConvProblem,
     [("nx", "nx"), ("ny", "ny"), ("nz", "nz"), ("in", "in_"), ("out", "out"), ("pre", "pre"),
      ("has_window", "has_window"), ("window", "window"), ("sums", "sums")]),
    ("steam_ba_problem_t", _lib.BAProblem,
     [("nx", "nx"), ("ny", "ny"), ("nz", "nz"), ("pert", "pert"), ("increment", "increment"),
      ("mean", "mean"), ("phi_min", "phi_min"), ("phi_max", "phi_max"),
      ("has_window", "has_window"), ("window", "window"), ("ledger", "ledger")]),
    ("steam_thermo_problem_t", _lib.ThermoProblem,
     [("nx", "nx"), ("ny", "ny"), ("nz", "nz"), ("h", "h"), ("qt", "qt"), ("prof", "prof"),
      ("compose", "compose"), ("bounds", "bounds"), ("surface_pressure", "surface_pressure"),
      ("ps_field", "ps_field"), ("T", "T"), ("qv", "qv"), ("qc", "qc"), ("qi", "qi"),
      ("p", "p")]),
]


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler on this host")
    lines = ['#include "steam_b200.h"', "#include <stddef.h>", "#include <stdio.h>",
             "int main(void) {"]
    for ctype, _, fields in STRUCTS:
        lines.append(f'  printf("{ctype} sizeof %zu\\n", sizeof({ctype}));')
        for cf, _ in fields:
            lines.append(f'  printf("{ctype} {cf} %zu\\n", offsetof({ctype}, {cf}));')
    lines += ["  return 0;", "}"]
    d = tmp_path_factory.mktemp("abi")
    src, exe = d / "abi.c", d / "abi"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run([cc, "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)],
                   check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    table = {}
    for line in out.splitlines():
        ctype, name, value = line.split()
        table[(ctype, name)] = int(value)
    return table


@pytest.mark.parametrize("ctype,cls,fields", STRUCTS, ids=[s[0] for s in STRUCTS])
def test_struct_layout_matches_header(c_layout, ctype, cls, fields):
    assert ctypes.sizeof(cls) == c_layout[(ctype, "sizeof")], ctype
    assert [f[0] for f in cls._fields_] == [pf for _, pf in fields], ctype
    for cf, pf in fields:
        assert getattr(cls, pf).offset == c_layout[(ctype, cf)], (ctype, cf)
