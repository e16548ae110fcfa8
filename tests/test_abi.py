"""The C-ABI libraries load and export every entry point that include/*.h
declares (no GPU needed: nothing is called)."""

import ctypes
import glob
import os
import re

import pytest

from polymage_b200 import headers
from polymage_b200.apps import catalog

INC = headers.INCLUDE


def declared(path):
    text = open(path).read()
    return re.findall(r'^\s*(?:void|int)\s+(pipeline_\w+)\s*\(', text, re.M)


def test_committed_headers_match_generated():
    exp = headers.expected_headers()
    for fn, text in exp.items():
        path = os.path.join(INC, fn)
        assert os.path.exists(path), fn
        assert open(path).read() == text, "%s is stale: run python -m " \
            "polymage_b200.headers" % fn


@pytest.mark.parametrize("name,builder", catalog.default_builds())
def test_library_exports_declared_symbols(name, builder):
    cp = builder().build()
    lib = ctypes.CDLL(cp.so_path)
    hdr = os.path.join(INC, "pipeline_%s.h" % cp.name)
    syms = declared(hdr)
    assert "pipeline_%s" % cp.name in syms and len(syms) >= 7
    for s in syms:
        assert hasattr(lib, s), s


def test_every_header_is_covered():
    names = set("pipeline_%s.h" % b().generate_code().name
                for _, b in catalog.default_builds())
    for path in glob.glob(os.path.join(INC, "pipeline_*.h")):
        assert os.path.basename(path) in names


def test_costmodel_library_exports_declared_symbols():
    from polymage_b200 import costmodel
    lib = costmodel.lib()
    text = open(os.path.join(INC, "pm_costmodel.h")).read()
    syms = re.findall(r'^\s*(?:long|int|void)\s+(pm_\w+)\s*\(', text, re.M)
    assert len(syms) >= 6
    for s in syms:
        assert hasattr(lib, s), s
