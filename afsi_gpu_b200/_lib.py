"""ctypes binding of ``libafsi_b200.so`` (the C-ABI in ``include/afsi_b200.h``).

PyTorch supplies device memory and the current CUDA stream; every compute call
goes to the native library.  There is no CPU or PyTorch fallback: a missing
library or a CPU tensor raises.
"""
import ctypes
import threading
from pathlib import Path
import torch

LIB_PATH = Path(__file__).resolve().parent / 'libafsi_b200.so'

F32, F64 = 0, 1
OK, ERR_ARG, ERR_CUDA = 0, 1, 2
FLAG_SUPPORT, FLAG_INDEX, FLAG_OVERFLOW, FLAG_TIMEOUT = 1, 2, 4, 8
PHI_CLAMPED, PHI_RADICAL = 0, 1
BC_NEUMANN, BC_CHANNEL, BC_PERIODIC, BC_DIRICHLET = 0, 1, 2, 3
MAX_LEVELS = 12

_lock = threading.Lock()
_lib = None

c_void_p, c_int64, c_int32, c_double = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_double
P_I64 = ctypes.POINTER(ctypes.c_int64)
P_F64 = ctypes.POINTER(ctypes.c_double)


class MGLevel(ctypes.Structure):
    _fields_ = [('shape', ctypes.c_int64 * 3), ('h2', ctypes.c_double * 3), ('inv_h2', ctypes.c_double * 3),
                ('p', c_void_p), ('ping', c_void_p), ('rhs', c_void_p)]


class MGPlan(ctypes.Structure):
    _fields_ = [('dim', c_int32), ('bc', c_int32), ('levels', c_int32), ('smooth', c_int32),
                ('dtype', c_int32), ('coarse_dtype', c_int32), ('level', MGLevel * MAX_LEVELS),
                ('coarse_inverse', c_void_p), ('scratch', c_void_p), ('smoother', c_int32)]


class PCGPlan(ctypes.Structure):
    _fields_ = [('crow', c_void_p), ('col', c_void_p), ('col32', c_void_p), ('val', c_void_p),
                ('diagonal', c_void_p), ('rhs', c_void_p), ('initial', c_void_p), ('x', c_void_p), ('r', c_void_p),
                ('d', c_void_p), ('Ad', c_void_p), ('state', c_void_p), ('scratch', c_void_p), ('rows', c_int64),
                ('cols', c_int32), ('dtype', c_int32), ('max_iterations', c_int32), ('check_every', c_int32),
                ('recompute_every', c_int32), ('diagonal_per_row', c_int32), ('rtol', ctypes.c_double),
                ('atol', ctypes.c_double)]


class RefineInstance(ctypes.Structure):
    _fields_ = [('nx', c_int64), ('ny', c_int64), ('h2', ctypes.c_double * 2), ('p', c_void_p), ('b', c_void_p),
                ('r32', c_void_p), ('e32', c_void_p)]


# name -> argtypes (restype int32 unless listed in _RESTYPES)
_SIGNATURES = {
    'afsi_b200_last_error': [],
    'afsi_b200_version': [],
    'afsi_b200_launch_count': [],
    'afsi_b200_compact_prepare': [c_void_p, c_int64, c_int32, P_F64, P_F64, P_F64, P_I64, c_int32, c_void_p,
                                  c_void_p, c_void_p, c_int32, c_void_p],
    'afsi_b200_indexed_prepare2d': [c_void_p, c_int64, c_int64, c_int64, c_double, c_double, c_double, c_double,
                                    c_void_p, c_void_p, c_void_p, c_int32, c_void_p],
    'afsi_b200_p2_prepare': [c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int64, P_F64, P_F64, P_F64,
                             c_void_p, c_void_p, c_int64, c_int64, c_void_p, c_int32, c_void_p],
    'afsi_b200_p2_orders': [c_void_p, c_int64, c_void_p, c_int64, ctypes.c_double, ctypes.c_double, c_int64,
                            c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_void_p],
    'afsi_b200_fe_prepare_mixed': [c_int32, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int64, P_F64, P_F64,
                                   P_F64, c_void_p, c_void_p, c_int64, c_int64, c_void_p, c_int32, c_void_p],
    'afsi_b200_det_plan_bytes': [c_int64, c_int64, c_int64, c_int64, c_int32],
    'afsi_b200_det_plan': [c_void_p, c_int64, c_int64, c_int64, c_int64, c_void_p, c_int64, c_void_p, c_int32,
                           c_void_p],
    'afsi_b200_det_spread': [c_void_p, c_void_p, c_void_p, c_int64, c_int64, c_int64, c_int64, c_void_p, c_int64,
                             c_void_p, c_void_p, c_void_p, c_int32, c_void_p],
    'afsi_b200_p2_point_forces': [c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int64, c_int64,
                                  ctypes.c_double, c_void_p, c_void_p, c_int32, c_void_p],
    'afsi_b200_p1_prepare': [c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int64, P_F64, P_F64, P_F64,
                             c_void_p, c_void_p, c_int64, c_int64, c_void_p, c_int32, c_void_p],
    'afsi_b200_p1_orders': [c_void_p, c_int64, c_void_p, c_int64, ctypes.c_double, ctypes.c_double, c_int64,
                            c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_void_p],
    'afsi_b200_p1_plan_scratch_bytes': [c_int64],
    'afsi_b200_p1_component_plan': [c_void_p, c_int64, c_int64, c_int64, c_int64, c_int32, c_int32, c_void_p,
                                    c_void_p, c_void_p, c_void_p, c_int64, c_void_p],
    'afsi_b200_hash_contract': [c_void_p] * 11 + [c_int64] * 5 + [c_int64, c_int32, c_int64, c_int64, c_int64,
                                                                    c_int32, c_int32, c_void_p],
    'afsi_b200_cached_contract': [c_void_p] * 11 + [c_int64, c_void_p, c_void_p, c_void_p, c_int64] +
                                 [c_int64] * 5 + [c_int32, c_int64, c_int64, c_int64, c_int32, c_int32, c_void_p],
    'afsi_b200_hash_accumulate': [c_void_p, c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_int64, c_int32,
                                  c_void_p],
    'afsi_b200_hash_csr_scratch_bytes': [c_int64, c_int32],
    'afsi_b200_hash_csr': [c_void_p, c_void_p, c_int64, c_int64, c_int64] + [c_void_p] * 8 + [c_int64, c_int32,
                                                                                             c_void_p],
    'afsi_b200_csr_spmv': [c_void_p, c_void_p, c_void_p, c_int64, c_int64, c_void_p, c_int64, c_void_p, c_int64,
                           ctypes.c_double, c_int32, c_void_p],
    'afsi_b200_mg_solve_graph_create': [ctypes.POINTER(MGPlan), c_int32, c_int32, c_void_p, c_void_p,
                                        ctypes.POINTER(c_void_p)],
    'afsi_b200_mg_solve_graph_create_started': [ctypes.POINTER(MGPlan), c_int32, c_int32, c_void_p, c_void_p,
                                                c_void_p, c_void_p, c_void_p, ctypes.POINTER(c_void_p)],
    'afsi_b200_mg_solve_graph_launch': [c_void_p, c_void_p],
    'afsi_b200_mg_solve_graph_destroy': [c_void_p],
    'afsi_b200_indexed_gather': [c_void_p, c_int64, c_int64, c_void_p, c_void_p, c_int64, c_int64, c_void_p,
                                 c_void_p, c_int32, c_void_p],
    'afsi_b200_indexed_spread': [c_void_p, c_int64, c_int64, c_void_p, c_void_p, c_int64, c_int64, c_double,
                                 c_void_p, c_void_p, c_int32, c_void_p],
    'afsi_b200_compact_gather': [c_void_p, c_void_p, c_void_p, c_int64, c_int64, c_int64, c_int64, c_void_p,
                                 c_void_p, c_int32, c_void_p],
    'afsi_b200_compact_spread': [c_void_p, c_void_p, c_void_p, c_int64, c_int64, c_int64, c_int64, c_double,
                                 c_void_p, c_void_p, c_int32, c_void_p],
    'afsi_b200_p2_spread': [c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_void_p, c_void_p,
                            c_int64, c_int64, c_void_p, c_void_p, c_void_p, c_int64, c_int64, c_int64, c_double,
                            c_void_p, c_int32, c_void_p],
    'afsi_b200_p2_gather_assemble': [c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_int64,
                                     c_void_p, c_void_p, c_void_p, c_int64, c_int64, c_void_p, c_int64, c_int64,
                                     c_int64, c_int64, c_void_p, c_int32, c_void_p],
    'afsi_b200_p2_gather_local': [c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_int64, c_void_p,
                                  c_void_p, c_void_p, c_int64, c_int64, c_void_p, c_int64, c_int64, c_int64,
                                  c_void_p, c_int32, c_void_p],
    'afsi_b200_node_reduce': [c_void_p, c_int64, c_void_p, c_void_p, c_int64, c_void_p, c_int32, c_void_p,
                              c_int32, c_void_p],
    'afsi_b200_mg_smooth': [c_void_p, c_void_p, c_void_p, P_I64, P_F64, P_F64, c_int32, c_int32, c_int32,
                            c_void_p],
    'afsi_b200_mg_residual': [c_void_p, c_void_p, c_void_p, P_I64, P_F64, c_int32, c_int32, c_int32, c_void_p],
    'afsi_b200_mg_restrict': [c_void_p, c_void_p, P_I64, c_int32, c_int32, c_void_p],
    'afsi_b200_mg_residual_restrict': [c_void_p, c_void_p, c_void_p, P_I64, P_F64, c_int32, c_int32, c_int32,
                                       c_void_p],
    'afsi_b200_mg_prolong_add': [c_void_p, c_void_p, P_I64, c_int32, c_int32, c_int32, c_void_p],
    'afsi_b200_mg_scratch_bytes': [ctypes.POINTER(MGPlan)],
    'afsi_b200_mg_vcycles': [ctypes.POINTER(MGPlan), c_int32, c_void_p],
    'afsi_b200_mg_residual_norm': [ctypes.POINTER(MGPlan), c_void_p, c_void_p],
    'afsi_b200_mg_residual_norm_noalloc': [c_void_p, c_void_p, P_I64, P_F64, c_int32, c_int32, c_void_p, c_int32,
                                           c_void_p],
    'afsi_b200_mg_sync_bytes': [],
    'afsi_b200_mg_persistent': [ctypes.POINTER(MGPlan), c_int32, c_int32, c_int32, c_double, c_void_p, c_void_p,
                                c_void_p],
    'afsi_b200_vector_stats': [c_void_p, c_int64, c_void_p, c_void_p, c_int32, c_void_p],
    'afsi_b200_subtract_mean': [c_void_p, c_int64, c_void_p, c_int32, c_void_p],
    'afsi_b200_mg_refine_scratch_bytes': [P_I64, c_int32, c_int32],
    'afsi_b200_mg_refine_residual': [c_void_p, c_void_p, c_void_p, P_I64, P_F64, c_int32, c_int32, c_void_p, c_void_p,
                                     c_void_p],
    'afsi_b200_mg_refine_correct': [c_void_p, c_void_p, c_int64, c_void_p],
    'afsi_b200_mg_batch_table_bytes': [c_void_p, c_int32],
    'afsi_b200_mg_batch_table': [c_void_p, c_int32, c_void_p, c_void_p, c_int64],
    'afsi_b200_mg_batch_vcycles': [c_void_p, c_int32, c_void_p, c_int32, c_int32, c_void_p],
    'afsi_b200_mg_batch_persistent': [c_void_p, c_int32, c_void_p, c_int32, c_int32, c_void_p, c_void_p],
    'afsi_b200_batch_refine_bytes': [c_void_p, c_int32],
    'afsi_b200_batch_refine_state_offset': [c_void_p, c_int32],
    'afsi_b200_batch_refine_setup': [c_void_p, c_int32, c_void_p, c_int64],
    'afsi_b200_batch_refine_start': [c_void_p, c_int32, c_void_p, c_double, c_double, c_int32, c_void_p],
    'afsi_b200_batch_refine_step': [c_void_p, c_int32, c_void_p, c_double, c_double, c_int32, c_void_p],
    'afsi_b200_batch_refine_graph_create': [c_void_p, c_int32, c_void_p, c_void_p, c_void_p, c_int32, c_double,
                                            c_double, c_int32, c_void_p],
    'afsi_b200_batch_refine_graph_launch': [c_void_p, c_void_p],
    'afsi_b200_batch_refine_graph_destroy': [c_void_p],
    'afsi_b200_fe_fused_spread': [c_int32, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_void_p, c_int64,
                                  c_void_p, c_void_p, P_F64, P_F64, P_F64, c_void_p, c_void_p, c_void_p, c_int64,
                                  c_int64, c_int64, c_double, c_void_p, c_int32, c_int32, c_void_p],
    'afsi_b200_fe_det_spread_bytes': [c_int64, c_int64, c_int64, c_int64, c_int32],
    'afsi_b200_fe_det_spread': [c_int32, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_void_p, c_int64,
                                c_void_p, c_void_p, P_F64, P_F64, P_F64, c_void_p, c_void_p, c_void_p, c_int64,
                                c_int64, c_int64, c_double, c_void_p, c_int64, c_void_p, c_int32, c_int32, c_void_p],
    'afsi_b200_fe_fused_gather': [c_int32, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_void_p, c_int64,
                                  c_void_p, c_void_p, c_void_p, c_void_p, P_F64, P_F64, P_F64, c_void_p, c_int64,
                                  c_int64, c_int64, c_void_p, c_int32, c_int32, c_void_p],
    'afsi_b200_fe_fused_gather_local': [c_int32, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_void_p, c_int64,
                                        c_void_p, c_void_p, c_void_p, c_void_p, P_F64, P_F64, P_F64, c_void_p,
                                        c_int64, c_int64, c_int64, c_void_p, c_int32, c_int32, c_void_p],
    'afsi_b200_stokes_packed_size': [P_I64],
    'afsi_b200_stokes_precondition_scratch_bytes': [P_I64],
    'afsi_b200_stokes_action': [c_void_p, c_void_p, P_I64, P_F64, c_double, c_double, c_int32, c_void_p],
    'afsi_b200_stokes_precondition_rhs': [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, P_I64, P_F64, c_double,
                                          c_int32, c_void_p],
    'afsi_b200_stokes_precondition_result': [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, P_I64,
                                             P_F64, c_double, c_double, c_int32, c_void_p],
    'afsi_b200_batch2d_prepare': [c_void_p, c_int64, c_void_p, c_int32, c_void_p, c_void_p, c_void_p, c_int32,
                                  c_void_p],
    'afsi_b200_batch2d_spread': [c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_int32, c_void_p, c_void_p,
                                 c_int64, c_int64, c_void_p, c_int32, c_void_p],
    'afsi_b200_batch2d_gather': [c_void_p, c_void_p, c_int64, c_int64, c_void_p, c_void_p, c_int64, c_void_p,
                                 c_void_p, c_int32, c_void_p],
    'afsi_b200_cache_scratch_bytes': [c_int64] * 5,
    'afsi_b200_cache_new_keys': [c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int64, c_int64, c_void_p, c_void_p,
                                 c_void_p, c_void_p, c_int64, c_void_p],
    'afsi_b200_cache_merge': [c_void_p, c_void_p, c_int64] + [c_void_p] * 4 + [c_int64, c_void_p, c_void_p, c_int64,
                                                                             c_int64, c_int64] +
                             [c_void_p] * 9 + [c_void_p, c_int64, c_int32, c_void_p],
    'afsi_b200_cache_values': [c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_int32, c_void_p],
    'afsi_b200_stokes_partial_blocks': [P_I64],
    'afsi_b200_helmholtz_initialize': [ctypes.POINTER(c_void_p), c_void_p, ctypes.POINTER(c_void_p), ctypes.POINTER(c_void_p), ctypes.POINTER(c_void_p), c_void_p, P_I64, P_F64, c_int32, c_void_p],
    'afsi_b200_helmholtz_sweep': [ctypes.POINTER(c_void_p), ctypes.POINTER(c_void_p), ctypes.POINTER(c_void_p), ctypes.POINTER(c_void_p), c_void_p, P_I64, P_F64, c_int32, c_void_p],
    'afsi_b200_stokes_start_partial': [ctypes.POINTER(c_void_p), c_void_p, c_void_p, P_I64, c_int32, c_void_p],
    'afsi_b200_stokes_residual_partial': [ctypes.POINTER(c_void_p), c_void_p, ctypes.POINTER(c_void_p), c_void_p, c_void_p, c_void_p, P_I64, c_int32,
                                          c_void_p],
    'afsi_b200_pressure_input_partial': [c_void_p, c_void_p, c_int64, c_void_p, c_int32, c_void_p],
    'afsi_b200_pressure_norm_partial': [c_void_p, c_void_p, c_void_p, c_void_p, P_I64, c_int32, c_void_p],
    'afsi_b200_pcg_scratch_bytes': [],
    'afsi_b200_pcg_begin': [ctypes.POINTER(PCGPlan), c_void_p],
    'afsi_b200_pcg_iterations': [ctypes.POINTER(PCGPlan), c_int32, c_void_p],
    'afsi_b200_pcg_graph_create': [ctypes.POINTER(PCGPlan), ctypes.POINTER(c_void_p)],
    'afsi_b200_pcg_graph_launch': [c_void_p, c_void_p],
    'afsi_b200_pcg_graph_destroy': [c_void_p],
}
_RESTYPES = {'afsi_b200_last_error': ctypes.c_char_p, 'afsi_b200_mg_scratch_bytes': ctypes.c_int64,
             'afsi_b200_mg_batch_table_bytes': ctypes.c_int64, 'afsi_b200_batch_refine_bytes': ctypes.c_int64,
             'afsi_b200_batch_refine_state_offset': ctypes.c_int64,
             'afsi_b200_stokes_packed_size': ctypes.c_int64,
             'afsi_b200_stokes_precondition_scratch_bytes': ctypes.c_int64,
             'afsi_b200_launch_count': ctypes.c_int64, 'afsi_b200_mg_sync_bytes': ctypes.c_int64,
             'afsi_b200_p1_plan_scratch_bytes': ctypes.c_int64, 'afsi_b200_hash_csr_scratch_bytes': ctypes.c_int64,
             'afsi_b200_pcg_scratch_bytes': ctypes.c_int64, 'afsi_b200_mg_refine_scratch_bytes': ctypes.c_int64,
             'afsi_b200_stokes_partial_blocks': ctypes.c_int64, 'afsi_b200_cache_scratch_bytes': ctypes.c_int64,
             'afsi_b200_det_plan_bytes': ctypes.c_int64, 'afsi_b200_fe_det_spread_bytes': ctypes.c_int64}


def exported_symbols():
    """Names every build of the library must export (declared in the header)."""
    return tuple(_SIGNATURES)


def load():
    """Load (building first if absent) and return the ctypes library."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                from .build import build
                build()
            lib = ctypes.CDLL(str(LIB_PATH))
            for name, args in _SIGNATURES.items():
                fn = getattr(lib, name)
                fn.argtypes = args
                fn.restype = _RESTYPES.get(name, ctypes.c_int32)
            _lib = lib
    return _lib


def call(name, *args):
    """Invoke an entry point; raise RuntimeError on a host status != 0."""
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != OK:
        msg = lib.afsi_b200_last_error().decode(errors='replace')
        raise RuntimeError(f'{name}: {msg}' if msg else f'{name} failed with status {rc}')
    return rc


def dtype_code(dtype):
    if dtype == torch.float64:
        return F64
    if dtype == torch.float32:
        return F32
    raise ValueError('IB/MG kernels support float32/float64')


def ptr(t):
    return None if t is None else t.data_ptr()


def stream(device=None):
    return torch.cuda.current_stream(device).cuda_stream


def doubles(values):
    values = [float(v) for v in values]
    return (ctypes.c_double * len(values))(*values)


def pointers(tensors):
    """Device pointers of three face arrays as a `void* const*` argument."""
    return (c_void_p * 3)(*[t.data_ptr() for t in tensors])


def int64s(values):
    values = [int(v) for v in values]
    return (ctypes.c_int64 * len(values))(*values)


def require_cuda(tensor):
    """Native kernels only: CPU tensors are rejected, never handled on the CPU."""
    if not torch.is_tensor(tensor) or not tensor.is_cuda:
        raise ValueError('the B200 backend requires CUDA tensors; there is no CPU fallback')
    load()


_status = {}


def status_word(device):
    """Int32 status word that kernels OR their AFSI_FLAG_* bits into, one per
    device and current stream, so that work on different streams (threads of
    a server, say) never clears or reads another's flags."""
    index = torch.device(device).index if torch.device(device).index is not None else torch.cuda.current_device()
    key = (index, torch.cuda.current_stream(index).cuda_stream)
    word = _status.get(key)
    if word is None:
        word = torch.zeros((), dtype=torch.int32, device=torch.device('cuda', index))
        _status[key] = word
    return word


_replayed = [0]


def launch_count():
    """Native kernel launches so far, including those replayed from captured graphs."""
    return int(load().afsi_b200_launch_count()) + _replayed[0]


def count_replay(launches):
    _replayed[0] += int(launches)


def forget_launches(launches):
    """Take back launches that were only captured into a graph, not run."""
    _replayed[0] -= int(launches)
