"""rusty_h264_b200 -- the encoder pixel hot path of rusty_h264 on B200 (sm_100a).

The product is libh264accel_cuda.so (C ABI, include/h264accel.h); this package
holds its Python binding (:mod:`accel`) and the seeded synthetic clips used for
benchmarking (:mod:`synth`).
"""
from .accel import (Accel, AccelError, METRIC_SAD, METRIC_SAD_AVG, METRIC_SATD, METRIC_SATD_AVG,
                    METRIC_SATD_WELS, default_me_params, frame_lambda, load_library, mv_cost_table,
                    split_gate_for_qp)

__all__ = [
    "Accel", "AccelError", "METRIC_SAD", "METRIC_SAD_AVG", "METRIC_SATD", "METRIC_SATD_AVG", "METRIC_SATD_WELS",
    "default_me_params", "frame_lambda", "load_library", "mv_cost_table", "split_gate_for_qp",
]
