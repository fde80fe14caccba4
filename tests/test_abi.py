"""The C-ABI library loads on a machine without a GPU, exports every entry point include/opensol_fdtd.h declares,
and rejects invalid configurations with OS_ERR_INVALID and a message before touching the device."""
import ctypes
import os
import re

import pytest

from opensol_b200 import _native
from opensol_b200.build import LIB_DIR, LIB_NAME, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for fname in os.listdir(os.path.join(ROOT, 'include')):
        if fname.endswith('.h'):
            text = open(os.path.join(ROOT, 'include', fname)).read()
            names |= set(re.findall(r'\b(os_\w+)\s*\(', text))
    return names


@pytest.fixture(scope='module')
def lib():
    build(verbose=False)
    return _native.load()


def test_every_declared_symbol_is_exported(lib):
    declared = _declared()
    assert declared, 'no declarations found'
    missing = [name for name in sorted(declared) if not hasattr(lib, name)]
    assert not missing, f'declared but not exported: {missing}'


def test_binding_signatures_cover_the_header():
    assert _declared() == set(_native.SIGNATURES), 'ctypes signatures and header declarations differ'


def test_version(lib):
    assert lib.os_fdtd_version() >= 100


@pytest.mark.parametrize('grid,match', [
    ((0, 10, 0, 0, 10, 15, 0), 'no cells'),
    ((20, 20, 0, 0, 10, 15, 0), 'cannot hold'),
    ((100, 100, 1, 0, 10, 15, 0), 'must be paired'),
    ((100, 100, 0, 0, 0, 15, 0), 'cpml_npml'),
    ((100, 100, 0, 0, 10, 64, 0), 'beyond the 2D faces'),
])
def test_create_rejects_invalid_grid(lib, grid, match):
    g = _native.OsGrid2D(*grid)
    h = ctypes.c_void_p()
    rc = lib.os_fdtd2d_create(ctypes.byref(g), ctypes.byref(h))
    assert rc == _native.OS_ERR_INVALID
    assert h.value is None
    assert re.search(match, _native.last_error())
    with pytest.raises(ValueError, match=match):
        _native.check(rc)


def test_null_handle_calls_fail_cleanly(lib):
    assert lib.os_fdtd2d_advance(None, 1, None, 0, 0, None) == _native.OS_ERR_INVALID
    assert lib.os_fdtd2d_destroy(None) == _native.OS_OK
    assert 'null handle' in _native.last_error()


def test_library_lives_in_tree():
    assert os.path.dirname(_native.LIB_PATH) == LIB_DIR and _native.LIB_PATH.endswith(LIB_NAME)
    assert LIB_DIR.startswith(ROOT)
