"""ctypes binding of libmi3b200.so (the C ABI declared in include/mi3b200.h).

The library is loaded from the package directory.  There is no fallback:
if the shared library is missing or fails to load, every call raises.
"""
import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libmi3b200.so"

c = ctypes
_vp, _u32, _u64, _f32, _i32 = c.c_void_p, c.c_uint32, c.c_uint64, c.c_float, c.c_int32

# name -> (restype, argtypes); mirrors include/mi3b200.h
SIGNATURES = {
    "mi3_last_error": (c.c_char_p, []),
    "mi3_abi_version": (c.c_int, []),
    "mi3_probe_bounded_wait": (c.c_int, [_vp, _u64, _u64, _vp, _vp]),
    "mi3_init_rng": (c.c_int, [_vp, _u32, _u64, _u64, _vp]),
    "mi3_jrows_stride": (_u64, [_u32, _u32]),
    "mi3_unpack_j": (c.c_int, [_vp, _vp, _u32, _u32, _vp]),
    "mi3_metropolis": (c.c_int, [_vp, _vp, _u32, _vp, _u32, _vp, _f32, _vp, _u32, _u32, _u32, _vp, _vp]),
    "mi3_metropolis_plan": (c.c_int, [_vp, _vp, _u32, _vp, _u32, _vp, _f32, _vp, _u32, _u32, _u32, _u32, _u32,
                                      _u32, _vp, _vp]),
    "mi3_metropolis_plans": (_u32, [_u32, _u32, _u32, _vp, _u32]),
    "mi3_jtiles_floats": (_u64, [_u32, _u32]),
    "mi3_unpack_j_tiles": (c.c_int, [_vp, _vp, _u32, _u32, _vp]),
    "mi3_metropolis_skew": (c.c_int, [_vp, _vp, _u32, _vp, _u32, _vp, _f32, _vp, _u32, _u32, _u32, _u32, _u32, _vp,
                                      _vp]),
    "mi3_gen_indep": (c.c_int, [_vp, _u32, _u32, _vp, _vp, _u32, _u32, _vp]),
    "mi3_energies_workspace": (c.c_size_t, [_u32]),
    "mi3_energies": (c.c_int, [_vp, _vp, _u32, _u32, _vp, _u32, _u32, _vp, c.c_size_t, _vp]),
    "mi3_energies_noalloc": (c.c_int, [_vp, _vp, _u32, _u32, _vp, _u32, _u32, _vp]),
    "mi3_energies_tc": (c.c_int, [_vp, _vp, _u32, _u32, _vp, _u32, _u32, _vp, c.c_size_t, _vp, _vp]),
    "mi3_energies_cons_workspace": (c.c_size_t, [_u32, _u32, _u32]),
    "mi3_energies_cons": (c.c_int, [_vp, _vp, _u32, _u32, _vp, _u32, _u32, _vp, _vp, c.c_size_t, _vp]),
    "mi3_rank_workspace": (c.c_size_t, [_u32]),
    "mi3_rank_average": (c.c_int, [_vp, _u32, _vp, _vp, c.c_size_t, _vp]),
    "mi3_rank_corr_workspace": (c.c_size_t, []),
    "mi3_rank_corr": (c.c_int, [_vp, _vp, _u32, _vp, _vp, c.c_size_t, _vp]),
    "mi3_equil_decide": (c.c_int, [_vp, _vp, c.c_double, _vp, _vp]),
    "mi3_bicounts": (c.c_int, [_vp, _u32, _u32, _vp, _u32, _u32, _vp]),
    "mi3_bicounts_tc_plan": (_u32, [_u32, _u32, _u32, _vp]),
    "mi3_bicounts_tc": (c.c_int, [_vp, _u32, _u32, _vp, _u32, _u32, _vp, _vp]),
    "mi3_bicounts_to_bimarg": (c.c_int, [_vp, _vp, _u32, _u32, _u32, _vp]),
    "mi3_weighted_marg_workspace": (c.c_size_t, [_u32, _u32, _u32]),
    "mi3_weighted_marg": (c.c_int, [_vp, _vp, _u32, _u32, _vp, _u32, _u32, _vp, _vp, c.c_size_t, _vp]),
    "mi3_weighted_marg_tc_workspace": (c.c_size_t, [_u32, _u32]),
    "mi3_weighted_marg_tc": (c.c_int, [_vp, _vp, _u32, _u32, _vp, _u32, _u32, _vp, c.c_size_t, _vp, _vp]),
    "mi3_copy_subseq": (c.c_int, [_vp, _u32, _u32, _vp, _vp, _u32, _u32, _vp]),
    "mi3_seqs_to_text": (c.c_int, [_vp, _u32, _u32, _u32, c.c_char_p, _u32, _vp, _vp, _vp]),
    "mi3_text_to_seqs": (c.c_int, [_vp, _u32, _u32, _u32, _u32, c.c_char_p, _u32, _vp, _u32, _u32, _vp, _vp]),
    "mi3_site_consensus_workspace": (c.c_size_t, [_u32, _u32]),
    "mi3_site_consensus": (c.c_int, [_vp, _u32, _u32, _u32, _u32, _vp, _vp, c.c_size_t, _vp]),
    "mi3_renormalize_bimarg": (c.c_int, [_vp, _u32, _u32, _vp]),
    "mi3_repack_seqs_T": (c.c_int, [_vp, _u32, _vp, _u32, _u32, _vp]),
    "mi3_update_j": (c.c_int, [_vp, _vp, _f32, _f32, _vp, _vp, _u32, _u32, _vp]),
    "mi3_reg_l1z": (c.c_int, [_vp, _f32, _f32, _f32, _vp, _vp, _u32, _u32, _vp]),
    "mi3_reg_l2z": (c.c_int, [_vp, _f32, _f32, _f32, _vp, _vp, _u32, _u32, _vp]),
    "mi3_reg_scadj": (c.c_int, [_vp, _f32, _f32, _f32, _f32, _vp, _vp, _u32, _u32, _vp]),
    "mi3_reg_x": (c.c_int, [_vp, _f32, _f32, _f32, _vp, _vp, _u32, _u32, _vp]),
    "mi3_reg_xij": (c.c_int, [_vp, _vp, _f32, _f32, _vp, _vp, _u32, _u32, _vp]),
    "mi3_reg_scadx": (c.c_int, [_vp, _f32, _f32, _f32, _f32, _f32, _vp, _vp, _u32, _u32, _vp]),
    "mi3_reg_expx": (c.c_int, [_vp, _f32, _f32, _f32, _vp, _vp, _u32, _u32, _vp]),
    "mi3_reg_dde": (c.c_int, [_vp, _f32, _f32, _f32, _vp, _vp, _u32, _u32, _vp]),
    "mi3_reg_scaddde": (c.c_int, [_vp, _f32, _f32, _f32, _f32, _vp, _vp, _u32, _u32, _vp]),
    "mi3_min_floats": (c.c_int, [_vp, _u32, _vp, _vp]),
    "mi3_dE_to_weights": (c.c_int, [_f32, _vp, _vp, _u32, _vp]),
    "mi3_fixed_beta_weights": (c.c_int, [_f32, _f32, _vp, _vp, _u32, _vp]),
    "mi3_weight_stats_workspace": (c.c_size_t, [_u32]),
    "mi3_weight_stats": (c.c_int, [_vp, _u32, _vp, _vp, _vp, c.c_size_t, _vp]),
    "mi3_weights_fused": (c.c_int, [_f32, _vp, _vp, _u32, _vp, _vp, _vp, _vp, c.c_size_t, _vp]),
    "mi3_add_float_bufs": (c.c_int, [_vp, _vp, _u32, _vp]),
    "mi3_weights_fused_dev": (c.c_int, [_vp, _vp, _vp, _u32, _vp, _vp, _vp, _vp, c.c_size_t, _vp]),
    "mi3_capture_begin": (c.c_int, [_vp]),
    "mi3_capture_end": (c.c_int, [_vp, c.POINTER(_vp)]),
    "mi3_graph_instantiate": (c.c_int, [_vp, c.POINTER(_vp)]),
    "mi3_graph_launch": (c.c_int, [_vp, _vp]),
    "mi3_graph_destroy": (c.c_int, [_vp, _vp]),
    "mi3_capture_while_begin": (c.c_int, [_vp, _vp, c.POINTER(c.c_ulonglong)]),
    "mi3_capture_while_end": (c.c_int, [_vp]),
    "mi3_newton_control": (c.c_int, [c.c_ulonglong, _vp, _vp, _vp, _vp, _vp, c.c_double, _vp, _vp]),
    "mi3_newton_adapt": (c.c_int, [_u32, _vp, _vp, _vp, _vp, _u32, _vp]),
    "mi3_memset": (c.c_int, [_vp, c.c_int, c.c_size_t, _vp]),
    "mi3_stream_create": (c.c_int, [c.POINTER(_vp)]),
    "mi3_stream_destroy": (c.c_int, [_vp]),
    "mi3_gauge_workspace": (c.c_size_t, [_u32, _u32]),
    "mi3_gauge_fieldless_even": (c.c_int, [_vp, _vp, _u32, _u32, _vp, c.c_size_t, _vp]),
    "mi3_bimarg_stats_workspace": (c.c_size_t, [_u32]),
    "mi3_bimarg_stats": (c.c_int, [_vp, _vp, _vp, _u32, _u32, _vp, _vp, c.c_size_t, _vp]),
    "mi3_made_forward": (c.c_int, [_vp, _u32, _u32, _u32, _u32, _u32, _u32] + [_vp] * 12 + [_vp]),
    "mi3_made_backward": (c.c_int, [_vp, _u32, _u32, _u32, _u32, _u32, _u32] + [_vp] * 21 + [_vp]),
    "mi3_made_adam": (c.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _u64, _f32, _f32, _f32, _f32, _u32, _vp]),
    "mi3_made_round_bf16": (c.c_int, [_vp, _vp, _vp, _u64, _vp]),
    "mi3_made_sample": (c.c_int, [_u32, _u32, _u32] + [_vp] * 8 + [_vp, _u32, _u32, _vp, _u64, c.c_int32, _vp]),
    "mi3_mh_independence": (c.c_int, [_vp, _vp, _u32, _u32, _u32, _vp, _vp, _vp, _vp, _u64, _vp, _vp]),
    "mi3_cond_handle_create": (c.c_int, [_vp, _u32, c.POINTER(c.c_ulonglong)]),
    "mi3_capture_if_begin": (c.c_int, [_vp, _vp, c.c_ulonglong]),
    "mi3_capture_if_end": (c.c_int, [_vp]),
    "mi3_equil_control": (c.c_int, [c.c_ulonglong, c.c_int32, _vp, _vp, c.c_double, c.c_int32, _u32, _u32, _u32,
                                    _vp, _vp]),
    "mi3_made_gemm_workspace": (_u64, [_u32, _u32, _u32, _u32]),
    "mi3_made_forward_tc": (c.c_int, [_vp, _u32, _u32, _u32, _u32, _u32, _u32] + [_vp] * 12 + [_vp, _u64, _vp, _vp]),
    "mi3_made_backward_tc": (c.c_int, [_vp, _u32, _u32, _u32, _u32, _u32, _u32] + [_vp] * 21 + [_vp, _u64, _vp, _vp]),
    "mi3_gemm_bf16_workspace": (_u64, [_u32, _u32, _u32]),
    "mi3_gemm_bf16": (c.c_int, [_u32, _u32, _u32, _vp, c.c_int64, c.c_int64, _vp, c.c_int64, c.c_int64, _vp,
                                c.c_int64, _f32, _f32, _vp, _u64, _vp, _vp]),
    "mi3_made_tc_workspace": (_u64, [_u32, _u32, _u32, _u32, _vp, _vp]),
    "mi3_made_tc_prepare": (c.c_int, [_u32, _u32, _u32, _u32] + [_vp] * 8 + [_vp, _u64, _vp, _vp]),
    "mi3_made_tc_sample": (c.c_int, [_vp, _vp, _u32, _u32, _vp, _u64, c.c_int32, _vp, _vp]),
}


class Mi3Error(RuntimeError):
    """A libmi3b200 call returned an error code."""

    def __init__(self, name, code, msg):
        super().__init__(f"{name} failed ({code}): {msg}")
        self.code = code


_lib = None


def load():
    """Load the shared library (raises if it is missing or incomplete)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"libmi3b200.so not built at {LIB_PATH}; run python -m mi3gpu_b200.build")
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def call(name, *args):
    """Call an int-returning entry point; raise Mi3Error on a negative code."""
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != 0:
        msg = lib.mi3_last_error().decode(errors="replace")
        raise Mi3Error(name, rc, msg)
    return rc


def query(name, *args):
    """Call a value-returning entry point (sizes, strides)."""
    return getattr(load(), name)(*args)
