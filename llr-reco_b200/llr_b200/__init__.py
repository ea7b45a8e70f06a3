"""B200-native LLR diffusion-MRI reconstruction: Python host side of libllr_b200.so.

The CUDA library is mapped on first use of a name that needs it (``import llr_b200`` alone
loads nothing), so pure-numpy helpers such as ``llr_b200.phantom`` can be imported by code that
must not map the library.  Every binding still goes through ``_lib``, which raises if the
library is missing: there is no CPU fallback.
"""
import importlib

_FROM_LIB = ("LLR_FORWARD", "LLR_INVERSE", "LLR_PROX_HARD_RANK", "LLR_PROX_SOFT_THRESH", "LIB_PATH", "LlrError",
             "check", "lib")
_FROM_API = ("DeviceBuffer", "PinnedBuffer", "ReconContext", "ReconParams", "cu_dwt_denoise",
             "cu_low_rank_approx_batch", "daubechies_filters", "device_count", "dti_back_project", "dti_project",
             "lift_data_set", "rand_shift", "signal_model", "to_ref_layout", "un_lift_data_set", "vd_mask")

__all__ = list(_FROM_LIB + _FROM_API)


def __getattr__(name):
    if name in _FROM_LIB:
        mod = importlib.import_module("._lib", __name__)
    elif name in _FROM_API:
        mod = importlib.import_module(".api", __name__)
    else:
        raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
    value = getattr(mod, name)
    globals()[name] = value
    return value
