"""ctypes binding of libopensol_fdtd.so (the C ABI of include/opensol_fdtd.h).

The library is loaded from the package's own ``_lib`` folder.  There is no fallback: a missing library, a missing
symbol or a machine without a CUDA device raises, so the B200 kernels are the only path that ever computes.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, '_lib', 'libopensol_fdtd.so')

OS_OK, OS_ERR_INVALID, OS_ERR_CUDA, OS_ERR_NO_MEMORY, OS_ERR_STATE = 0, 1, 2, 3, 4
OS_SIDE_BITS = {'x_lo': 1, 'x_hi': 2, 'y_lo': 4, 'y_hi': 8, 'z_lo': 16, 'z_hi': 32}
OS_EZ, OS_HX, OS_HY = 0, 1, 2
OS_HZ_HZ, OS_HZ_EX, OS_HZ_EY = 0, 1, 2   # field buffers of an H_z engine
FIELDS_3D = ('ex', 'ey', 'ez', 'hx', 'hy', 'hz')   # os_fdtd3d_read_field / write_field component order

_lock = threading.Lock()
_lib = None


class OsGrid2D(ctypes.Structure):
    _fields_ = [('nx', ctypes.c_int32), ('ny', ctypes.c_int32), ('periodic_x', ctypes.c_int32),
                ('periodic_y', ctypes.c_int32), ('npml', ctypes.c_int32), ('cpml_sides', ctypes.c_int32),
                ('device', ctypes.c_int32)]


class OsGrid3D(ctypes.Structure):
    _fields_ = [('nx', ctypes.c_int32), ('ny', ctypes.c_int32), ('nz', ctypes.c_int32),
                ('periodic', ctypes.c_int32 * 3), ('device', ctypes.c_int32)]


_F = ctypes.POINTER(ctypes.c_float)
_D = ctypes.POINTER(ctypes.c_double)
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_P = ctypes.c_void_p

# name -> argtypes (every entry point returns int); also the list the export test checks against the header.
SIGNATURES = {
    'os_fdtd_last_error': [ctypes.c_char_p, ctypes.c_size_t],
    'os_fdtd_version': [],
    'os_fdtd_pool_trim': [],
    'os_fdtd_host_alloc': [ctypes.c_size_t, ctypes.POINTER(_P)],
    'os_fdtd_host_free': [_P],
    'os_fdtd2d_create': [ctypes.POINTER(OsGrid2D), ctypes.POINTER(_P)],
    'os_fdtd2d_destroy': [_P],
    'os_fdtd2d_set_spacings': [_P, _F, _F, _F, _F],
    'os_fdtd2d_set_materials': [_P, _F, _F, _F, _F, ctypes.c_float, ctypes.c_float, ctypes.c_float],
    'os_fdtd2d_set_coefficients': [_P, _F, _F, _F, _F, ctypes.c_float, ctypes.c_float],
    'os_fdtd2d_read_cb': [_P, _F],
    'os_fdtd2d_hz_create': [ctypes.POINTER(OsGrid2D), ctypes.POINTER(_P)],
    'os_fdtd2d_hz_set_materials': [_P, _F, _F, _F, _F, _F, _F, _F, _F, _F, ctypes.c_float, ctypes.c_float,
                                   ctypes.c_float],
    'os_fdtd2d_hz_read_cb': [_P, _F, _F],
    'os_fdtd2d_hz_form': [_P, ctypes.POINTER(_I32)],
    'os_fdtd2d_hz_plan': [_P, ctypes.POINTER(_I64), ctypes.POINTER(_I64)],
    'os_fdtd2d_set_cpml_side': [_P, _I32, _F, _F, _F, _F, _F, _F],
    'os_fdtd2d_add_line_source': [_P, _I32, _I32, _I32, _I32, _F, ctypes.POINTER(_I32)],
    'os_fdtd2d_set_line_profile': [_P, _I32, _F],
    'os_fdtd2d_add_flux_line': [_P, _I32, _I32, _I32, _I32, _I32, ctypes.POINTER(_I32)],
    'os_fdtd2d_set_sample_interval': [_P, _I64],
    'os_fdtd2d_advance': [_P, _I64, _F, _I64, _I64, _F],
    'os_fdtd2d_advance_noalloc': [_P, _I64, _F, _I64, _I64, _F],
    'os_fdtd2d_step_count': [_P, ctypes.POINTER(_I64)],
    'os_fdtd2d_configure': [_P, _I32, _I32, _I32],
    'os_fdtd2d_launch_count': [_P, ctypes.POINTER(_I64)],
    'os_fdtd2d_set_profiling': [_P, _I32],
    'os_fdtd2d_autotune': [_P, _I32, ctypes.POINTER(_I32), _I32, _I32, ctypes.POINTER(_I32),
                           ctypes.POINTER(ctypes.c_float)],
    'os_fdtd2d_plan_info': [_P, _I32, ctypes.POINTER(_I64), ctypes.POINTER(_I64), ctypes.POINTER(_I64)],
    'os_fdtd2d_kernel_times': [_P, _I32, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_I64)],
    'os_fdtd2d_read_flux_spectra': [_P, _I32, _D, _D],
    'os_fdtd2d_add_dft_map': [_P, _I32, _I32, _I32, _I32, _I32, _I32, ctypes.POINTER(_I32)],
    'os_fdtd2d_read_dft_map': [_P, _I32, _F],
    'os_fdtd2d_add_probe': [_P, _I32, _I32, _I32, ctypes.POINTER(_I32)],
    'os_fdtd2d_add_pole': [_P, _I32, _I32, _I32, _I32, _I32, ctypes.c_float, ctypes.c_float, _F, ctypes.c_float,
                           ctypes.POINTER(_I32)],
    'os_fdtd2d_hz_add_pole': [_P, _I32, _I32, _I32, _I32, _I32, _I32, ctypes.c_float, ctypes.c_float, _F,
                              ctypes.c_float, ctypes.POINTER(_I32)],
    'os_fdtd2d_add_tfsf': [_P, _I32, _I32, _I32, _I32, _I32, _I32, _I32, _F, _F, ctypes.c_float, ctypes.c_float, _F, _F,
                           ctypes.POINTER(_I32)],
    'os_fdtd2d_read_probe': [_P, _I32, _F, _I64, ctypes.POINTER(_I64)],
    'os_fdtd2d_read_field': [_P, _I32, _F],
    'os_fdtd2d_write_field': [_P, _I32, _F],
    'os_fdtd2d_reset': [_P],
    'os_fdtd2d_synchronize': [_P],
    'os_fdtd2d_set_stream': [_P, _P],
    'os_fdtd2d_last_advance_ms': [_P, ctypes.POINTER(ctypes.c_float)],
    'os_fdtd2d_batch_create': [_I32, ctypes.POINTER(_P)],
    'os_fdtd2d_batch_destroy': [_P],
    'os_fdtd2d_batch_stream': [_P, ctypes.POINTER(_P)],
    'os_fdtd2d_batch_advance': [_P, ctypes.POINTER(_P), _I32, _I64, ctypes.POINTER(_F), ctypes.POINTER(_I64),
                                ctypes.POINTER(_I64), ctypes.POINTER(_F)],
    'os_fdtd2d_batch_last_ms': [_P, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(_I64)],
    'os_fdtd2d_adjoint_create': [_P, _I32, _I32, _I32, _I32, _I32, _I32, ctypes.POINTER(_P)],
    'os_fdtd2d_adjoint_destroy': [_P],
    'os_fdtd2d_adjoint_save': [_P, _I32],
    'os_fdtd2d_adjoint_reset': [_P],
    'os_fdtd2d_adjoint_segment': [_P, _I32, _I64, _I32, _F, _I32, _I32, ctypes.POINTER(_I32), _F, _F],
    'os_fdtd2d_adjoint_gradient': [_P, _D],
    'os_fdtd2d_set_stall_probe': [_P, _I64],
    'os_fdtd3d_create': [ctypes.POINTER(OsGrid3D), ctypes.POINTER(_P)],
    'os_fdtd3d_destroy': [_P],
    'os_fdtd3d_set_rows': [_P, _F, _F, _F, _F, _F, _F, _F],
    'os_fdtd3d_set_materials': [_P, ctypes.POINTER(ctypes.c_uint16), _I32, _F, _F, _F, _F, _F, _F, ctypes.c_float],
    'os_fdtd3d_set_cpml_axis': [_P, _I32, _I32, ctypes.POINTER(_I32), _F, _F, ctypes.POINTER(_I32), _F, _F],
    'os_fdtd3d_set_variant': [_P, _I32],
    'os_fdtd3d_set_fused_config': [_P, _I32],
    'os_fdtd3d_interior': [_P, ctypes.POINTER(_I32), ctypes.POINTER(_I32)],
    'os_fdtd3d_face_cb': [_P, _I32, _I32, _I32, _I32, _F],
    'os_fdtd3d_add_dipole': [_P, _I32, _I32, _I32, _I32, ctypes.c_float, ctypes.POINTER(_I32)],
    'os_fdtd3d_set_dipole_weight': [_P, _I32, ctypes.c_float],
    'os_fdtd3d_add_flux_monitor': [_P, _I32, ctypes.POINTER(_I32)],
    'os_fdtd3d_add_flux_pair': [_P, _I32, _I32, _I32, _I32, _I32, ctypes.POINTER(_I32), ctypes.POINTER(_I32),
                                ctypes.POINTER(_I32)],
    'os_fdtd3d_set_sample_interval': [_P, _I64],
    'os_fdtd3d_advance': [_P, _I64, _F, _I64, _I64, _F],
    'os_fdtd3d_read_field': [_P, _I32, _F],
    'os_fdtd3d_write_field': [_P, _I32, _F],
    'os_fdtd3d_read_flux_pair': [_P, _I32, _D, _D],
    'os_fdtd3d_reset': [_P],
    'os_fdtd3d_synchronize': [_P],
    'os_fdtd3d_set_stream': [_P, _P],
    'os_fdtd3d_set_x_chunk': [_P, _I32],
    'os_fdtd3d_last_advance_ms': [_P, ctypes.POINTER(ctypes.c_float)],
    'os_fdtd3d_launch_count': [_P, ctypes.POINTER(_I64)],
    'os_fdtd3d_step_count': [_P, ctypes.POINTER(_I64)],
}


class NativeError(RuntimeError):
    """A CUDA or device-state failure reported by libopensol_fdtd.so."""


def load():
    """The loaded library (built by ``python -m opensol_b200.build``); raises when it is missing."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f'{LIB_PATH} is not built; run `python -m opensol_b200.build` (the B200 CUDA '
                                   f'engine has no CPU fallback)')
            lib = ctypes.CDLL(LIB_PATH)
            for name, argtypes in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = ctypes.c_int
                fn.argtypes = argtypes
            _lib = lib
        return _lib


def last_error() -> str:
    lib = load()
    buf = ctypes.create_string_buffer(1024)
    lib.os_fdtd_last_error(buf, len(buf))
    return buf.value.decode('utf-8', 'replace')


def check(rc: int, what: str = '') -> None:
    """Raise the reference's exception type for a non-zero status: ValueError for a bad configuration, RuntimeError
    (NativeError) for CUDA / device-state failures, MemoryError for a failed device allocation."""
    if rc == OS_OK:
        return
    message = last_error() or what
    if rc == OS_ERR_INVALID:
        raise ValueError(message)
    if rc == OS_ERR_NO_MEMORY:
        raise MemoryError(message)
    raise NativeError(message)


def fptr(array):
    """float* of a C-contiguous float32 array (None -> NULL)."""
    if array is None:
        return None
    if array.dtype != np.float32 or not array.flags.c_contiguous:
        raise TypeError(f'expected a C-contiguous float32 array, got {array.dtype} contiguous={array.flags.c_contiguous}')
    return array.ctypes.data_as(_F)


def dptr(array):
    if array.dtype != np.float64 or not array.flags.c_contiguous:
        raise TypeError(f'expected a C-contiguous float64 array, got {array.dtype}')
    return array.ctypes.data_as(_D)


class _PinnedBlock:
    """Owner of one page-locked allocation; freed when the last array viewing it is collected."""

    def __init__(self, ptr):
        self.ptr = ptr

    def __del__(self):
        try:
            load().os_fdtd_host_free(self.ptr)
        except Exception:
            pass


def pinned_empty(shape, dtype=np.float32):
    """Uninitialised page-locked numpy array (os_fdtd_host_alloc); the allocation lives as long as the array."""
    dtype = np.dtype(dtype)
    count = int(np.prod(shape))
    ptr = ctypes.c_void_p()
    check(load().os_fdtd_host_alloc(count * dtype.itemsize, ctypes.byref(ptr)), 'os_fdtd_host_alloc')
    if count == 0:
        return np.empty(shape, dtype=dtype)
    raw = (ctypes.c_char * (count * dtype.itemsize)).from_address(ptr.value)
    array = np.frombuffer(raw, dtype=dtype).reshape(shape)
    owner = _PinnedBlock(ptr.value)
    # numpy keeps `raw` alive through the array's base chain; the owner rides on the ctypes buffer object
    raw._owner = owner
    return array
