"""Loads libreactive_b200.so and declares the C-ABI signatures.

The library is the product: there is no Python or CPU fallback. A missing or
unloadable library raises immediately.
"""
import ctypes as C
from pathlib import Path

from . import _abi as A

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libreactive_b200.so"

_d = C.POINTER(C.c_double)
_v = C.c_void_p
_s = C.POINTER(A.State)
_u64 = C.c_uint64

TRANSPORT = {
    "create": ([C.c_int, C.POINTER(A.Config), _d, C.POINTER(A.Face), _d, _s, _d, _d, C.c_char_p, C.c_size_t], _v),
    "create_v2": ([C.c_int, C.POINTER(A.Config), C.POINTER(A.OptionsV2), _d, C.POINTER(A.Face), _d, _s, _d, _d,
                   C.c_char_p, C.c_size_t], _v),
    "destroy": ([_v], None), "error": ([_v], C.c_char_p), "is_cuda": ([_v], C.c_int),
    "stats": ([_v, C.POINTER(A.Stats)], C.c_int),
    "profile": ([_v, C.POINTER(A.Profile)], C.c_int),
    "device_profile": ([_v, C.POINTER(A.DeviceProfile)], C.c_int),
    "memory_v2": ([_v, C.POINTER(A.MemoryV2)], C.c_int),
    "upload_conserved": ([_v, _d, _u64], C.c_int),
    "stable_step_primitives": ([_v, C.POINTER(A.Primitive), _s, C.c_double, C.c_double, _d], C.c_int),
    "stage_resident": ([_v, _s, _d, _d, C.c_double, C.c_int, _u64, _u64, _d, _d], C.c_int),
    "rhs": ([_v, _d, _s, _d, _d, _d, _d], C.c_int),
    "stage": ([_v, _d, _s, _d, _d, C.c_double, C.c_int, _d], C.c_int),
    "stable_step": ([_v, _d, _s, C.c_double, C.c_double, _d], C.c_int),
    "begin_attempt": ([_v, C.c_char_p, _u64], C.c_int),
    "end_attempt": ([_v, _u64, C.c_int], C.c_int),
    "advance_resident_v2": ([_v, A.Token, A.Token, _s, _v, _d, _d, C.c_double, _d], C.c_int),
    "download_conserved": ([_v, A.Token, _d], C.c_int),
    "set_wale_v1": ([_v, C.POINTER(A.WaleOptions)], C.c_int),
    "wale_profile_v1": ([_v, C.POINTER(A.WaleProfile)], C.c_int),
    "wale_primitives_v1": ([_v, C.POINTER(A.Primitive), _s, _d], C.c_int),
    "set_wale_scalars_v1": ([_v, C.POINTER(A.WaleScalarOptions)], C.c_int),
    "wale_scalar_profile_v1": ([_v, C.POINTER(A.WaleScalarProfile)], C.c_int),
    "wale_scalar_fields_v1": ([_v, _d, _d, _d, _d], C.c_int),
    "wale_scalar_fields_device_v3": ([_v, _v, _v, _v, _v, C.c_size_t, C.c_size_t, _v], C.c_int),
    "set_capillary_v1": ([_v, C.POINTER(A.CapillaryOptions)], C.c_int),
    "capillary_geometry_v1": ([_v, _d, _d, _d, _d, _d], C.c_int),
    "capillary_profile_v1": ([_v, C.POINTER(A.CapillaryProfile)], C.c_int),
    "set_wale_pr_model_v1": ([_v, C.POINTER(A.WalePrModel)], C.c_int),
    "wale_pr_properties_v1": ([_v, C.POINTER(A.WalePrEpoch), _d, C.c_size_t, _v], C.c_int),
    "wale_pr_properties_v2": ([_v, C.POINTER(A.WalePrEpoch), _d, C.c_size_t, _v, C.c_int], C.c_int),
    "wale_pr_profile_v1": ([_v, C.POINTER(A.WalePrProfile)], C.c_int),
    "capillary_resident_begin_v1": ([_v, C.c_size_t, _d, _d, _d, _v, _d, C.c_double, C.c_int, C.POINTER(C.c_int)],
                                    C.c_int),
    "capillary_resident_select_v1": ([_v, C.c_int, C.POINTER(A.CapillaryResidentView), C.POINTER(C.c_int)], C.c_int),
    "capillary_resident_update_v1": ([_v, C.c_size_t, _d, C.POINTER(C.c_int)], C.c_int),
    "capillary_resident_relax_v1": ([_v], C.c_int),
    "capillary_resident_commit_v1": ([_v, _v, _d, _d, _d], C.c_int),
    "layout_v3": ([_v, C.POINTER(C.c_size_t)] * 1 + [C.POINTER(C.c_size_t)] * 3, C.c_int),
    "fill_fixed_v3": ([_v, _v, _v, _v], C.c_int),
    "stage_device_v3": ([_v, _v, _v, _v, C.c_double, C.c_int, _v, _v], C.c_int),
    "stable_step_device_v3": ([_v, _v, _v, C.c_double, C.c_double, _v, _v], C.c_int),
    "stage_cfl_device_v3": ([_v, _v, _v, _v, C.c_double, C.c_int, _v, C.c_double, C.c_double, _v, _v], C.c_int),
    "status_v3": ([_v, C.POINTER(C.c_uint), C.c_int, _v], C.c_int),
    "structured_v3": ([_v, C.c_int, C.POINTER(C.c_int)], C.c_int),
    "precision_v3": ([_v, C.c_int, C.POINTER(C.c_int)], C.c_int),
    "flux_v3": ([_v, C.c_int, C.POINTER(C.c_int)], C.c_int),
    "autotune_v3": ([_v, _v, _v, _v, C.POINTER(C.c_uint)], C.c_int),
    "launch_shapes_v3": ([_v, _v, C.POINTER(C.c_uint)], C.c_int),
    "rate_vjp_v3": ([_v, _v, _v, _v, _v, _v, _v], C.c_int),
    "owned_cells_v3": ([_v, C.c_uint64, C.c_uint64], C.c_int),
}

HEM = {
    "numerical_policy_v1": ([], C.c_char_p),
    "create_v1": ([C.c_char_p, C.c_size_t, C.c_size_t, C.c_char_p, C.c_size_t], _v),
    "create_resident_v1": ([C.c_char_p, C.c_size_t, C.c_size_t, C.c_char_p, C.c_size_t], _v),
    "run_v2": ([_v, _d, _d, _v, C.c_size_t, _v, C.POINTER(C.c_int), C.POINTER(A.HemProfile), C.c_char_p, C.c_size_t],
               C.c_int),
    "run_resident_v1": ([_v, _v, _v, _v, _v, _v, C.c_size_t, _v, C.POINTER(A.HemProfile), C.c_char_p, C.c_size_t],
                        C.c_int),
    "initialize_tp_v1": ([_v, _d, _d, _v, C.c_size_t, _v, C.POINTER(C.c_int), C.POINTER(A.HemProfile), C.c_char_p,
                          C.c_size_t], C.c_int),
    "device_bytes_v1": ([_v], C.c_size_t),
    "destroy_v1": ([_v], None),
    "run_v1": ([_v, _d, _d, C.c_size_t, _v, C.POINTER(C.c_int), C.POINTER(A.HemProfile), C.c_char_p, C.c_size_t],
               C.c_int),
    "run_device_v3": ([_v, _v, C.c_size_t, C.c_size_t, C.c_size_t, _v, _v, _v, _v, _v, C.c_int, _v, C.c_char_p,
                       C.c_size_t], C.c_int),
    "run_counters_v3": ([_v, C.POINTER(A.HemProfile), _v, C.c_char_p, C.c_size_t], C.c_int),
    "two_phase_bound_v3": ([_v, C.c_int, C.POINTER(C.c_int), C.c_char_p, C.c_size_t], C.c_int),
    "vjp_device_v3": ([_v, _v, C.c_size_t, C.c_size_t, C.c_size_t, _v, _v, _v, C.c_size_t, _v, _v, C.c_char_p,
                       C.c_size_t], C.c_int),
    "autotune_v3": ([_v, _v, C.c_size_t, C.c_size_t, C.c_size_t, _v, _v, C.POINTER(C.c_int), C.c_char_p,
                     C.c_size_t], C.c_int),
}

_lib = None


IDEAL = {
    "create_v3": ([_v, C.c_size_t, C.c_double, C.c_double, C.c_double, C.c_char_p, C.c_size_t], _v),
    "destroy_v3": ([_v], None),
    "run_device_v3": ([_v, _v, C.c_size_t, C.c_size_t, C.c_size_t, _v, _v, _v, _v, _v, C.c_char_p, C.c_size_t],
                      C.c_int),
    "two_phase_bound_v3": ([_v, C.c_int, C.POINTER(C.c_int), C.c_char_p, C.c_size_t], C.c_int),
    "vjp_device_v3": ([_v, _v, C.c_size_t, C.c_size_t, C.c_size_t, _v, _v, _v, C.c_size_t, _v, C.c_char_p,
                       C.c_size_t], C.c_int),
}


MIXTURE = {
    "properties_v3": ([_v, C.c_size_t, _v, _v, _v, C.c_int, C.c_int, _v, _v, _v, _v, C.c_char_p, C.c_size_t],
                      C.c_int),
}


HOST = {
    "threads_v3": ([], C.c_int),
    "copy_v3": ([_v, _v, C.c_size_t], C.c_int),
    "transport_states_v3": ([_v, C.c_size_t, _d, C.c_size_t, C.c_size_t, _v, _v], C.c_int),
    "recovery_inputs_v3": ([_d, C.c_size_t, C.c_size_t, C.c_size_t, _d, _d], C.c_int),
}


def load():
    """The loaded library with typed entry points (raises if it is absent)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run __graft_entry__.build() (the CUDA library is required)")
        lib = C.CDLL(str(LIB_PATH))
        for table, prefix in ((TRANSPORT, "reactive_transport_"), (HEM, "reactive_gpu_hem_"),
                              (IDEAL, "reactive_ideal_gas_"), (MIXTURE, "reactive_b200_mixture_"),
                              (HOST, "reactive_b200_host_")):
            for name, (args, ret) in table.items():
                fn = getattr(lib, prefix + name, None)
                if fn is None:
                    continue
                fn.argtypes, fn.restype = args, ret
        _lib = lib
    return _lib
