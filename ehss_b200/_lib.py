"""ctypes binding of libehss_b200.so (the C ABI in include/ehss_b200.h).

The CUDA library is the only implementation of the path: there is no CPU
fallback.  ``load()`` raises when the shared library is missing or cannot be
loaded; callers that need the GPU get a clear error instead of a silent
substitute.
"""
from __future__ import annotations

import ctypes as ct
import re
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / 'libehss_b200.so'
HEADER = HERE.parent / 'include' / 'ehss_b200.h'

OK, ERR_VALUE, ERR_CUDA, ERR_CAPACITY, ERR_DEVICE = 0, 1, 2, 3, 4
PREC_FP64, PREC_FP32 = 0, 1
STAT_BOX, STAT_SPHERE, STAT_QUERIES, STAT_GRAZING, STAT_FALLBACK, STAT_FP64, STAT_ERRORS = range(7)
NSTATS = 8
BLOCK_EHSS, BLOCK_PA = 1, 2
LAUNCH_COUNT_TESTS = 1
LAUNCH_RAY_BLOCKS = 2
LAUNCH_NO_DISK_BLOCKS = 4
# LBVH leaf bound used by default: leaves of 13-16 atoms trace fastest on B200 with the default launch
DEFAULT_LEAF = 14
BUILD_EXTERIOR = 1
BLOCK_RAYS = 4
FX_SCALE = 2.0 ** -36

P = ct.c_void_p
I32, I64, U64 = ct.c_int32, ct.c_int64, ct.c_uint64


class SceneInfo(ct.Structure):
    _fields_ = [('n_atoms', I64), ('n_nodes', I64), ('leaf_size', I32), ('depth', I32),
                ('center', ct.c_double * 3), ('radius', ct.c_double), ('scale', ct.c_double),
                ('rmax', ct.c_double), ('bytes', U64), ('n_active', I64), ('exterior', I32), ('reserved', I32)]


class Block(ct.Structure):
    _fields_ = [('basis', (ct.c_uint32 * 4) * 30), ('base', ct.c_uint32 * 4), ('scene', P), ('log2_rays', I32),
                ('cap', I32), ('precision', I32), ('flags', ct.c_uint32), ('hist_offset', I64),
                ('chunk_begin', I64), ('rays', P), ('ray_scale', ct.c_double), ('reserved', I64)]


class BlockResult(ct.Structure):
    _fields_ = [('angle_fx', U64), ('hits', U64), ('unresolved', U64), ('escaped', U64), ('pa_blocked', U64),
                ('hits_fx', U64), ('unresolved_fx', U64), ('pa_fx', U64), ('stats', U64 * NSTATS)]


class Residual(ct.Structure):
    _fields_ = [('o', ct.c_double * 3), ('d', ct.c_double * 3), ('din', ct.c_double * 3), ('block', I32),
                ('last_rank', I32), ('bounces', I32), ('reserved', I32)]


class Extension(ct.Structure):
    _fields_ = [('angle_fx', U64), ('escaped', U64), ('unresolved', U64), ('continued', U64)]


class Boundary(ct.Structure):
    _fields_ = [('kind', I32), ('reserved', I32), ('center', ct.c_double * 3), ('rotation', ct.c_double * 9),
                ('axes', ct.c_double * 3)]


class Launch(ct.Structure):
    _fields_ = [('block_threads', I32), ('ctas_per_sm', I32), ('chunk_rays', I32), ('resolve_batch', I32),
                ('precisions', I32), ('options', I32), ('smem_stack', I32), ('reserved', I32)]


_SIGNATURES = {
    'ehss_last_error': (ct.c_char_p, []),
    'ehss_abi_version': (ct.c_int, []),
    'ehss_sobol_scramble': (ct.c_int, [ct.c_int, U64, P, P]),
    'ehss_sobol_points': (ct.c_int, [ct.c_int, U64, I64, I64, P, P]),
    'ehss_scene_bytes': (ct.c_int, [I64, ct.c_int, P, P]),
    'ehss_scene_build': (ct.c_int, [I64, P, P, ct.c_int, P, U64, P, U64, P]),
    'ehss_scene_build_noalloc': (ct.c_int, [I64, P, P, ct.c_int, P, U64, P]),
    'ehss_scenes_workspace_bytes': (ct.c_int, [ct.c_int, P, P]),
    'ehss_scenes_build': (ct.c_int, [ct.c_int, P, P, P, ct.c_int, P, P, P, U64, P]),
    'ehss_scenes_build_ex': (ct.c_int, [ct.c_int, P, P, P, ct.c_int, P, P, P, U64, ct.c_uint32, P]),
    'ehss_enclosing_radius': (ct.c_int, [I64, P, P, P]),
    'ehss_scenes_refit': (ct.c_int, [ct.c_int, P, P, P, P, P, U64, P]),
    'ehss_scene_info_get': (ct.c_int, [P, P, P]),
    'ehss_source_rays': (ct.c_int, [P, ct.c_int, U64, I64, I64, P, P, P]),
    'ehss_compact_source_rays': (ct.c_int, [P, ct.c_int, U64, I64, I64, P, P, P, P]),
    'ehss_trace': (ct.c_int, [P, I64, ct.c_int, ct.c_int, P, P, P, P, P, P, P, P, P]),
    'ehss_pa_anyhit': (ct.c_int, [P, I64, P, P, P, P, P, P]),
    'ehss_pa_grid_workspace_bytes': (ct.c_int, [I64, ct.c_int, ct.c_int, P]),
    'ehss_pa_grid': (ct.c_int, [P, I64, ct.c_int, U64, ct.c_int, P, P, P, P, U64, P]),
    'ehss_blocks_prepare': (ct.c_int, [P, ct.c_int, P, ct.c_int, P]),
    'ehss_blocks_workspace_bytes': (ct.c_int, [ct.c_int, P]),
    'ehss_trace_blocks': (ct.c_int, [P, ct.c_int, I64, P, P, P, I64, P, U64, P, P]),
    'ehss_trace_blocks_residual': (ct.c_int, [P, ct.c_int, I64, P, P, P, I64, P, U64, P, P, I64, P, P]),
    'ehss_trace_blocks_window': (ct.c_int, [P, ct.c_int, I64, I64, I64, P, P, P, I64, P, U64, P, P]),
    'ehss_extend_blocks': (ct.c_int, [P, ct.c_int, P, ct.c_int, P, I64, ct.c_int, P, P, P, P, I64, P, P, P]),
}

_LIB = None


class EHSSDeviceError(RuntimeError):
    pass


def load():
    """Load (building first if absent) the CUDA library; raise if impossible."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        try:
            from . import build as _build
            _build.build()
        except Exception as exc:  # no nvcc, or compilation failed
            raise RuntimeError(f'libehss_b200.so is missing and could not be built: {exc}') from exc
    lib = ct.CDLL(str(LIB_PATH))
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.ehss_abi_version() != 1:
        raise RuntimeError('libehss_b200.so ABI mismatch')
    _LIB = lib
    return lib


def check(rc, what=''):
    if rc == OK:
        return
    msg = load().ehss_last_error().decode(errors='replace')
    text = f'{what}: {msg}' if what else msg
    if rc == ERR_VALUE:
        raise ValueError(text)
    if rc == ERR_CAPACITY:
        raise MemoryError(text)
    raise EHSSDeviceError(text)


def header_functions():
    """Function names declared in include/ehss_b200.h."""
    text = HEADER.read_text()
    return sorted(set(re.findall(r'^\s*(?:int|const char\*)\s+(ehss_\w+)\s*\(', text, flags=re.M)))
