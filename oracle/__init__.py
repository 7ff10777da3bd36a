"""CPU oracle of the in-place cut-rank DP executor (TEST INFRASTRUCTURE ONLY; see oracle.py)."""
from .oracle import Oracle, build, host_has_avx512, ref_binary, ref_gpu_binary, ref_isa, run_ref, uniforms  # noqa: F401
from . import statevector  # noqa: F401
