"""nb6b200 -- B200-native force hot path of Nbody6++GPU behind its C ABI.

The product is ``libnb6b200.so`` (CUDA, sm_100a) next to this package.  This
module loads it and exposes it through :class:`nb6b200.abi.ForceLib`, the
numpy-level mirror of the reference's ``gpunb_*`` / ``gpupot_`` /
``irr_simd_*`` calls.  There is no CPU fallback: if the shared object is
missing, :func:`load` raises.
"""
from __future__ import annotations

import ctypes as C
import os

from .abi import ForceLib

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "libnb6b200.so")

# Every extern "C" symbol the library exports (declared in include/nb6b200.h).
ABI_SYMBOLS = (
    "gpunb_devinit_", "gpunb_open_", "gpunb_close_", "gpunb_send_", "gpunb_regf_",
    "gpunb_profile_",
    "gpupot_",
    "irr_simd_open_", "irr_simd_close_", "irr_simd_profile_", "irr_simd_set_jp_",
    "irr_simd_set_list_", "irr_simd_firr_vec_",
    "gpuirr_open_", "gpuirr_close_", "gpuirr_set_jp_", "gpuirr_set_list_",
    "nb6_set_abort_on_error_", "nb6_last_status_", "nb6_device_",
    "nb6_regf_device_", "nb6_regf_outputs_", "nb6_regf_last_kernel_ms_", "nb6_regf_tune_",
    "nb6_regf_last_geometry_", "nb6_regf_autotune_", "nb6_regf_tuned_", "nb6_regf_graphs_", "nb6_regf_jsort_", "nb6_regf_seg_",
    "nb6_irr_predict_send_", "nb6_irr_last_kernel_ms_", "nb6_regf_proposals_",
    "nb6_hermite_open_", "nb6_hermite_set_", "nb6_irr_correct_", "nb6_regf_correct_", "nb6_hermite_get_", "nb6_ks_set_", "nb6_blocks_run_", "nb6_blocks_mode_", "nb6_irr_tune_", "nb6_irr_pv_", "nb6_blocks_active_", "nb6_blocks_regular_",
    "nb6_mlp_size_", "nb6_mlp_init_", "nb6_mlp_set_", "nb6_mlp_get_", "nb6_mlp_grad_",
    "nb6_mlp_train_", "nb6_mlp_predict_", "nb6_mlp_enable_",
    "nb6_sync_", "nb6_stream_",
    "nb6_pot_device_", "nb6_pot_last_kernel_ms_",
    "nb6_state_open_", "nb6_state_set_", "nb6_state_update_", "nb6_predict_",
    "nb6_predict_device_", "nb6_predict_send_", "nb6_predict_last_kernel_ms_",
    "nb6_state_close_",
    "nb6_fp32_peak_probe_",
    "nb6_regf_noalloc_",
    "nb6_hermite_adjust_", "nb6_irr_lists_get_",
)

_LIB: C.CDLL | None = None


def library_path() -> str:
    return LIB_PATH


def load_cdll() -> C.CDLL:
    """Load libnb6b200.so (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with "
                "`python nbody6ppgpu-beijing_b200/build.py` (there is no CPU fallback)")
        _LIB = C.CDLL(LIB_PATH, mode=C.RTLD_LOCAL)
        _LIB.nb6_last_status_.restype = C.c_int
        _LIB.nb6_device_.restype = C.c_int
        _LIB.nb6_regf_last_kernel_ms_.restype = C.c_float
        _LIB.nb6_stream_.restype = C.c_void_p
        if hasattr(_LIB, "nb6_pot_last_kernel_ms_"):
            _LIB.nb6_pot_last_kernel_ms_.restype = C.c_float
        if hasattr(_LIB, "nb6_fp32_peak_probe_"):
            _LIB.nb6_fp32_peak_probe_.restype = C.c_double
        if hasattr(_LIB, "nb6_predict_last_kernel_ms_"):
            _LIB.nb6_predict_last_kernel_ms_.restype = C.c_float
        if hasattr(_LIB, "nb6_irr_last_kernel_ms_"):
            _LIB.nb6_irr_last_kernel_ms_.restype = C.c_float
    return _LIB


def load() -> ForceLib:
    return ForceLib(load_cdll(), name="libnb6b200")


def set_abort_on_error(flag: bool) -> None:
    load_cdll().nb6_set_abort_on_error_(C.byref(C.c_int(1 if flag else 0)))


def last_status() -> int:
    return int(load_cdll().nb6_last_status_())


__all__ = ["ForceLib", "load", "load_cdll", "library_path", "ABI_SYMBOLS",
           "set_abort_on_error", "last_status"]
