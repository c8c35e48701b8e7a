"""Python host side of the B200 batched MuJoCo step.

The product is the C-ABI library libmjb200.so (include/mjmlx/*.h); this
package binds it with ctypes and mirrors the reference's Python interface
(python/rl_bindings.cpp: BatchedSim.step(ctrl, n), state(), set_state()).
"""
from .capi import lib, load_model, load_model_from_string, Model, BatchedSim, WarmStart, gemm_bf16, parse_dump  # noqa: F401
from . import models  # noqa: F401
