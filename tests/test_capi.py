"""The C ABI: the library loads without a GPU and exports every symbol that
include/bfgt.h declares; calls that need a device fail with a status, not a
crash."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import heat2d_per_box_b200 as hb
from heat2d_per_box_b200 import _lib

from conftest import has_gpu

HEADER = Path(__file__).resolve().parents[1] / "include" / "bfgt.h"


def declared_symbols():
    src = HEADER.read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", src)
    skip = {"if", "while", "for", "sizeof", "return"}
    return sorted({n for n in names if n not in skip and (n.startswith("bfgt_") or n == "boxfgt_")})


def test_header_symbols_exported():
    L = C.CDLL(str(_lib.lib_path() if _lib.lib_path().exists() else _lib.lib()._name))
    syms = declared_symbols()
    assert "boxfgt_" in syms and "bfgt_plan_execute" in syms
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_no_torch_types_in_header():
    src = HEADER.read_text()
    assert "torch" not in src.lower().replace("no torch", "")
    assert "at::" not in src


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_plan_without_device_reports_status():
    g = np.array([[0.1, 0.2, 0.07, 0.5]])
    t = hb.build_uniform(2, g, norder=8)
    with pytest.raises(hb.BfgtError) as e:
        hb.Plan(t, 1e-3, 1e-9)
    assert e.value.code == 6  # BFGT_ERR_NODEVICE


def test_boxfgt_rejects_unsupported_flags():
    g = np.array([[0.1, 0.2, 0.07, 0.5]])
    t = hb.build_uniform(2, g, norder=8)
    pot = np.zeros(t.nboxes * t.npbox)
    ti = np.zeros(20)
    with pytest.raises(hb.BfgtError, match="ndim=2"):
        hb.boxfgt(1, 3, 1e-3, 1e-9, 0, 1, 8, 64, t.nboxes, t.nlevels, t.ltree, t.itree.copy(), t.iptr, t.centers,
                  t.boxsize, t.fvals, 1, pot, None, None, 0, 0, None, 0, None, None, None, ti)
    with pytest.raises(hb.BfgtError, match="grad/hess"):      # ifpgh=2 needs a grad array
        hb.boxfgt(1, 2, 1e-3, 1e-9, 0, 1, 8, 64, t.nboxes, t.nlevels, t.ltree, t.itree.copy(), t.iptr, t.centers,
                  t.boxsize, t.fvals, 2, pot, None, None, 0, 0, None, 0, None, None, None, ti)
    with pytest.raises(hb.BfgtError, match="ifpgh=1,2,3"):
        hb.boxfgt(1, 2, 1e-3, 1e-9, 0, 1, 8, 64, t.nboxes, t.nlevels, t.ltree, t.itree.copy(), t.iptr, t.centers,
                  t.boxsize, t.fvals, 4, pot, None, None, 0, 0, None, 0, None, None, None, ti)
    with pytest.raises(hb.BfgtError, match="ifnewtree=0"):
        hb.boxfgt(1, 2, 1e-3, 1e-9, 0, 1, 8, 64, t.nboxes, t.nlevels, t.ltree, t.itree.copy(), t.iptr, t.centers,
                  t.boxsize, t.fvals, 1, pot, None, None, 1, 0, None, 0, None, None, None, ti)
    assert not pot.any()


def test_default_precision_and_plan_cache_api():
    """The drop-in's precision selector and plan-cache queries need no device."""
    hb.set_default_precision(hb.BFGT_PREC_SPLIT)
    hb.set_default_precision(hb.BFGT_PREC_FP64)
    with pytest.raises(hb.BfgtError):
        hb.set_default_precision(7)
    hb.plan_cache_clear()
    info = hb.plan_cache_info()
    assert info["entries"] == 0 and info["capacity"] >= 0
    b = hb.last_call_bytes()
    assert set(b) == {"h2d", "d2h"} and min(b.values()) >= 0
