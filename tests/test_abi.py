"""The C ABI: the native library loads without a GPU and exports every entry
point include/fornax_b200.h declares."""
import ctypes
import os
import re

import pytest

from tests.conftest import ROOT

HEADER = os.path.join(ROOT, "include", "fornax_b200.h")


def declared():
    text = open(HEADER).read()
    return re.findall(r"^\s*(?:int|void|fx_shard_group\s*\*)\s*(fx_\w+)\s*\(", text, re.M)


def test_header_declares_entry_points():
    names = declared()
    assert len(names) >= 25
    assert len(set(names)) == len(names)


def test_library_exports_every_declared_symbol():
    from fornaxamr_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"
    assert set(_lib.EXPORTS) == set(declared())


def test_struct_layout_matches_header():
    from fornaxamr_b200._lib import FxBlockDesc, FxConfig, FxSlot
    assert ctypes.sizeof(FxSlot) == 24
    assert ctypes.sizeof(FxBlockDesc) == 16 + 13 * 8 + 56 * 24 + 10 * 4
    assert ctypes.sizeof(FxConfig) == 8 + 8 + 48 + 24 + 8 + 8 + 8
    from fornaxamr_b200._lib import FxAmrConfig, FxAmrCriterion
    assert ctypes.sizeof(FxAmrCriterion) == 16 + 24
    assert ctypes.sizeof(FxAmrConfig) == 24 + 24 + 4 * 40


def test_invalid_arguments_are_rejected_without_device():
    import fornaxamr_b200 as fx
    L = fx.library()
    cfg = fx.make_config(True, 5.0 / 3.0, (0, 1, 0, 1, 0, 1))
    cfg.gamma = -1.0
    h = ctypes.c_void_p()
    assert L.fx_create(0, ctypes.byref(cfg), ctypes.byref(h)) == fx._lib.FX_EINVAL
    assert L.fx_create(0, None, ctypes.byref(h)) == fx._lib.FX_EINVAL


def test_plan_export_rejects_non_outflow_field_boundaries():
    import fornaxamr_b200 as fx
    from fornaxamr_b200 import mesh
    blocks = mesh.uniform_mesh((2, 1, 1), (0, 1, 0, 0.5, 0, 0.5))
    desc = mesh.to_desc(blocks)
    cfg = fx.make_config(True, 5.0 / 3.0, (0, 1, 0, 0.5, 0, 0.5), bc=(1, 0, 0, 0, 0, 0))
    with pytest.raises(fx.FxError):
        fx.plan_export(cfg, desc, 1)
