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
