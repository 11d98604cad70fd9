"""The C-ABI library builds, loads and exports what include/kielflow_b200.h declares."""
import ctypes
import os
import re

import pytest

import kielflow_b200 as kf
from kielflow_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "kielflow_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\w[\w\s\*]*?\b(kf_\w+)\s*\(", text, re.M)))


def test_header_declares_the_binding_exports():
    assert set(declared_symbols()) == set(_lib.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = _lib.load_library()
    for sym in declared_symbols():
        assert hasattr(lib, sym), sym


def test_context_creation_fails_loudly_without_a_b200():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    cfg = kf.Config.make(16, 25.1, 0.8)
    with pytest.raises(kf.KfError) as e:
        kf.Context(cfg)
    assert e.value.code in (-5, -2)


def test_config_layout_matches_header():
    text = open(HEADER).read()
    body = text[text.index("typedef struct {"):text.index("} kf_config;")]
    names = re.findall(r"\b(?:int|double)\s+(\w+);", body)
    assert names == [f for f, _ in kf.Config._fields_]


def test_grid_mirror_axes():
    """interfaces.Grid: axis_CoEqSt and the sine-stretched axis_CoSiSt positions
    (the restatement's, which match the reference's), dS and the config it
    hands to the contexts."""
    import math

    import numpy as np

    from kielflow_b200 import inputs as I
    from kielflow_b200.interfaces import Grid
    from oracle import bind

    L = I.L_DEFAULT
    m = I.frontend_stretch(L)
    for mm in (0.0, m):
        g = Grid(16, L, mm)
        o = bind.Oracle(bind.config(16, L, 1.0, stretch_m=mm))
        assert np.array_equal(np.array([g.val_at(i) for i in range(-1, 17)]), o.positions())
        assert g.type_id == (3 if mm else 1)
    g = Grid(16, L, m)
    assert abs(g.dS(8) - 0.3) < 1e-15 and abs(g.dS(0) - 1.7) < 1e-15
    assert abs(sum(g.dS(i) for i in range(16)) * (L / 16) - L) < 1e-12
    with pytest.raises(ValueError):
        Grid(16, L, L / (2.0 * math.pi))


def test_struct_layouts_match_the_header(tmp_path):
    """sizeof and every field offset of the C ABI's structs, compiled from
    include/kielflow_b200.h with the host C compiler, against the ctypes mirrors."""
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    mirrors = {"kf_config": _lib.Config, "kf_diag_out": _lib.DiagOut, "kf_grad_out": _lib.GradOut,
               "kf_tune_out": _lib.TuneOut, "kf_output": _lib.Output, "kf_file_info": _lib.FileInfo}
    lines = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append(f'printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c99", "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            s, f, v = line.split()
            got[(s, f)] = int(v)
    for cname, py in mirrors.items():
        assert got[(cname, "sizeof")] == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)
