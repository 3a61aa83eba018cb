"""ecg_b200 -- B200 (sm_100a, FP64) drop-in for the variational hot path of
ATOM-MOL-nonBO: ECG pair elements, H/S assembly, the LDL^H inverse-iteration
solve of HC = ESC and the nonlinear-parameter gradient, behind the C ABI of
include/ecg_abi.h.  This package is the Python mirror of that ABI."""
from .system import System, expand_yhy, parse_young, transposition_matrix
from .context import Context, EcgError, probe_fp64_peak, probe_fp64_tensor_peak
from . import synth, inout, expc

__all__ = ["System", "Context", "EcgError", "probe_fp64_peak", "probe_fp64_tensor_peak", "expand_yhy", "parse_young", "transposition_matrix", "synth", "inout", "expc"]
