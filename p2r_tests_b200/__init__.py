"""p2r-b200: B200-native (sm_100a) helix propagation + Kalman update over Matriplex arrays.

The package `p2r-tests_b200` is spelled `p2r_tests_b200` because Python module names
cannot contain '-'. The compute path is libp2r_b200.so (hand-written CUDA behind the C ABI
in include/p2r.h); this package is the Python host side over that ABI.
"""
from ._lib import (FLAG_ADJ_FP32, FLAG_FP32_DET, FLAG_NO_STAGING, FLAG_ORDER_BY_LAYERS, FLAG_SQUASH_PHI, MODE_CHAINED, MODE_RESTART, P2RError, LIB_PATH, lib)
from .api import (Config, KalmanGain, KalmanGainInv, KalmanUpdate, REF_BZ, count_nonfinite, forward, forward_host, fp32_fma_probe, fp64_fma_probe, gen_params,
                  generate_fixture,
                  generate_helix, generate_helix_device, kfact, math_check, math_variant, propagateToR, run_layers, summary, tracks_cov, tracks_par, tracks_q)

from .autograd import P2RChain, auto_ckpt_stride, forward_backward, workspace_size
from .uneven import (Queue, inverse, inverse_device, lognormal_counts, permute_tracks, permute_tracks_device, plan,
                     sort_by_layers, sort_by_layers_device, uneven_workload)
from . import autotune

__all__ = [
    "P2RChain", "auto_ckpt_stride", "forward_backward", "workspace_size", "Queue", "lognormal_counts", "plan", "uneven_workload", "sort_by_layers", "sort_by_layers_device", "permute_tracks", "permute_tracks_device", "inverse", "inverse_device",
    "Config", "KalmanGain", "KalmanGainInv", "KalmanUpdate", "propagateToR", "run_layers", "forward", "forward_host", "fp32_fma_probe", "fp64_fma_probe",
    "count_nonfinite", "kfact", "math_check", "math_variant",
    "gen_params", "generate_helix", "generate_helix_device", "generate_fixture", "summary", "tracks_par", "tracks_cov", "tracks_q",
    "MODE_CHAINED", "MODE_RESTART", "FLAG_ADJ_FP32", "FLAG_FP32_DET", "FLAG_NO_STAGING", "FLAG_ORDER_BY_LAYERS", "FLAG_SQUASH_PHI", "P2RError", "REF_BZ", "LIB_PATH", "lib",
]
