"""sqdft_b200: SQDFT's spectral-quadrature step on NVIDIA B200 (sm_100a).

The CUDA library behind ``include/sqdft_b200.h`` computes the SQ electron
density, band / entropy energies and nonlocal forces; this package is its
Python host mirror (``sq``), the case-file reader (``case``) and the build
step (``build``).
"""
from .case import Case, load_case, read_container, save_case, write_container  # noqa: F401

__all__ = ["Case", "load_case", "save_case", "read_container", "write_container"]
