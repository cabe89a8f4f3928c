"""ctypes binding of the isw C ABI (include/isw.h). The library is built in-tree (build.py) and must exist: there is no
fallback of any kind, so a missing or stale library is an ImportError."""
import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get('ISW_LIB', HERE / 'libisw.so'))

ISW_OK, ISW_EINVAL, ISW_ECUDA, ISW_ENOMEM, ISW_EUNSUPPORTED, ISW_ETIMEOUT, ISW_ENOTFINITE = range(7)
ISW_FP64, ISW_MIXED = 0, 1

if not LIB_PATH.exists():
    raise ImportError(f'isw: {LIB_PATH} is missing; build it with python insilica-world-v2_b200/build.py')
lib = ctypes.CDLL(str(LIB_PATH))

P, I, D, LL = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_longlong


class GridHost(ctypes.Structure):
    _fields_ = [('n', I), ('N', I), ('E', I), ('NV', I),
                ('eI', P), ('eJ', P), ('nbr', P), ('cellEdge', P), ('cellEdgeAsc', P), ('cellSign', P), ('ev1', P), ('ev2', P),
                ('vEdge', P), ('vCell', P), ('vEdgeSign', P), ('vSlot', P), ('eoeStart', P), ('eoe', P),
                ('le', P), ('de', P), ('areaCell', P), ('areaV', P), ('fV', P), ('kite', P), ('w', P),
                ('deg', P), ('dist', P), ('eKi', P), ('eKj', P)]


class LayersParams(ctypes.Structure):
    _fields_ = [('L', I), ('grav', D), ('gprime', P), ('drag', P), ('stress', P),
                ('nu4', D), ('floor_', D), ('rotation', D), ('div_damp', D), ('thin', D), ('vmix', D), ('vmix_cd', D),
                ('b', P), ('precision', I), ('air', I), ('cp', D), ('kappa', D), ('rd', D), ('p0', D),
                ('thin_wind', D), ('wall', P), ('shelf', D), ('shelf_bed', I),
                ('percall', I)]


def _sig(name, res, args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = args
    return f


isw_last_error = _sig('isw_last_error', ctypes.c_char_p, [])
isw_version = _sig('isw_version', I, [])
isw_grid_create = _sig('isw_grid_create', I, [ctypes.POINTER(GridHost), I, ctypes.POINTER(P)])
isw_grid_destroy = _sig('isw_grid_destroy', I, [P])
isw_layers_create = _sig('isw_layers_create', I, [P, ctypes.POINTER(LayersParams), ctypes.POINTER(P)])
isw_layers_destroy = _sig('isw_layers_destroy', I, [P])
isw_layers_step = _sig('isw_layers_step', I, [P, P, P, P, D, I, P])
isw_layers_step_air = _sig('isw_layers_step_air', I, [P, P, P, P, P, D, I, P])
isw_layers_update_gfast = _sig('isw_layers_update_gfast', I, [P, P, P, P])
isw_layers_exchange = _sig('isw_layers_exchange', I, [P, P, P, P, P, P, P, I, P])
isw_layers_set_option = _sig('isw_layers_set_option', I, [P, I, P, D])
ISW_OPT_SIG, ISW_OPT_TIDE, ISW_OPT_CBOT, ISW_OPT_CD_BOT = 1, 2, 3, 4
isw_layers_substeps = _sig('isw_layers_substeps', I, [P, P, D, ctypes.POINTER(I), P])
isw_layers_lap = _sig('isw_layers_lap', I, [P, P, P, P])
isw_layers_vmix_heat = _sig('isw_layers_vmix_heat', I, [P, P, P, P, D, D, D, D, P])
isw_layers_mask = _sig('isw_layers_mask', I, [P, P, I, P])
isw_layers_status = _sig('isw_layers_status', I, [P, P, I])
isw_layers_set_bottom = _sig('isw_layers_set_bottom', I, [P, P, P])
isw_transport_create = _sig('isw_transport_create', I, [P, I, D, I, I, ctypes.POINTER(P)])
isw_transport_destroy = _sig('isw_transport_destroy', I, [P])
isw_transport_mass_after = _sig('isw_transport_mass_after', I, [P, P, P, P, P])
isw_transport_step_many = _sig('isw_transport_step_many', I, [P, P, P, P, ctypes.POINTER(P), I, I, P])
isw_dsum = _sig('isw_dsum', I, [P, P, LL, ctypes.POINTER(D), P])
isw_dsum_static = _sig('isw_dsum_static', I, [P, P, LL, P, P])
isw_mesh_build = _sig('isw_mesh_build', I, [I, I, I, I, P, ctypes.POINTER(P)])
isw_mesh_get = _sig('isw_mesh_get', I, [P, ctypes.c_char_p, ctypes.POINTER(P), ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(I)])
isw_mesh_destroy = _sig('isw_mesh_destroy', I, [P])
isw_batch_create = _sig('isw_batch_create', I, [I, ctypes.POINTER(P)])
isw_batch_destroy = _sig('isw_batch_destroy', I, [P])
isw_batch_add = _sig('isw_batch_add', I, [P, P, P, P, P, P, P, P, ctypes.POINTER(P), I, D, I, ctypes.POINTER(I)])
isw_batch_add_air = _sig('isw_batch_add_air', I, [P, P, P, P, P, P, P, P, P, ctypes.POINTER(P), I, D, I, ctypes.POINTER(I)])
isw_batch_remove = _sig('isw_batch_remove', I, [P, I])
isw_batch_step = _sig('isw_batch_step', I, [P, P])
isw_batch_config = _sig('isw_batch_config', I, [P, I, I, I, I, I])
isw_batch_info = _sig('isw_batch_info', I, [P, ctypes.POINTER(I), ctypes.POINTER(I), ctypes.POINTER(I), ctypes.POINTER(LL),
                                             ctypes.POINTER(I), ctypes.POINTER(I)])
isw_batch_pipeline = _sig('isw_batch_pipeline', I, [P, I])
isw_batch_grid_loop = _sig('isw_batch_grid_loop', I, [P, I])
isw_batch_level_layout = _sig('isw_batch_level_layout', I, [P, I, I, I, I])
isw_batch_flush = _sig('isw_batch_flush', I, [P, P])
isw_batch_status = _sig('isw_batch_status', I, [P, P, I])
isw_batch_fault_test = _sig('isw_batch_fault_test', I, [P, LL, P])


class IswError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f'isw status {status}: {msg}')
        self.status = status


def check(status):
    if status != ISW_OK:
        msg = isw_last_error().decode(errors='replace')
        if status == ISW_EUNSUPPORTED:
            raise NotImplementedError(msg)
        if status == ISW_EINVAL:
            raise ValueError(msg)
        raise IswError(status, msg)


def host_ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def host_array(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)
