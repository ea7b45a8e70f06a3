"""B200-native LLR diffusion-MRI reconstruction: Python host side of libllr_b200.so."""
from ._lib import (LLR_FORWARD, LLR_INVERSE, LLR_PROX_HARD_RANK, LLR_PROX_SOFT_THRESH, LIB_PATH, LlrError,
                   check, lib)
from .api import (DeviceBuffer, PinnedBuffer, ReconContext, ReconParams, cu_dwt_denoise, cu_low_rank_approx_batch,
                  daubechies_filters, device_count, dti_back_project, dti_project, lift_data_set, rand_shift,
                  signal_model, to_ref_layout, un_lift_data_set, vd_mask)

__all__ = [
    "LLR_FORWARD", "LLR_INVERSE", "LLR_PROX_HARD_RANK", "LLR_PROX_SOFT_THRESH", "LIB_PATH", "LlrError", "check",
    "lib", "DeviceBuffer", "PinnedBuffer", "ReconContext", "ReconParams", "cu_dwt_denoise",
    "cu_low_rank_approx_batch", "daubechies_filters", "device_count", "dti_back_project", "dti_project",
    "lift_data_set", "rand_shift", "signal_model", "to_ref_layout", "un_lift_data_set", "vd_mask",
]
