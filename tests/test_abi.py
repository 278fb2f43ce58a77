"""The C-ABI library builds, loads without a GPU, and exports every declared symbol."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in ("rgsplat.h", "rgsplat_debug.h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(rgs_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from rgsplat_b200 import build

    build.build()
    return ctypes.CDLL(build.LIB)


def test_headers_declare_entry_points():
    names = declared_functions()
    assert "rgs_render_and_backward" in names and "rgs_trainer_step" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"missing exports: {missing}"


def test_python_binding_covers_every_symbol():
    from rgsplat_b200 import _lib

    missing = [n for n in declared_functions() if n not in _lib.SIGNATURES]
    assert not missing, f"ctypes signatures missing: {missing}"


def test_defaults_without_gpu(lib):
    from rgsplat_b200 import _lib

    L = _lib.load()
    o = _lib.rgs_options()
    L.rgs_options_default(ctypes.byref(o))
    assert (o.tile_w, o.tile_h, o.batch, o.reference_compat, o.exact_loss) == (16, 16, 256, 1, 0)
    c = _lib.rgs_train_config()
    L.rgs_train_config_default(ctypes.byref(c))
    assert abs(c.lr_position - 0.00016) < 1e-9 and c.max_gaussians == 3_000_000
    assert c.densify_from_iter == 500 and c.opacity_reset_iter == 3000


def test_struct_layouts():
    from rgsplat_b200 import _lib

    assert ctypes.sizeof(_lib.rgs_camera) == 4 * (2 + 4 + 16 + 3)
    assert ctypes.sizeof(_lib.rgs_splat_info_2d) == 40
    assert ctypes.sizeof(_lib.rgs_train_config) == 96
