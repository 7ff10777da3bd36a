"""CPU oracle of the in-place cut-rank DP executor (TEST INFRASTRUCTURE ONLY; see oracle.py)."""
from .oracle import Oracle, build, ref_binary, run_ref, uniforms  # noqa: F401
from . import statevector  # noqa: F401
