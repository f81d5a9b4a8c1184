"""B200 sliding-window backend solver (CGMLI-SLAM ``backend_visual_batch: schur`` path).

The compute path is the CUDA library ``lib/libcgmli_backend.so`` behind the C
ABI of ``include/cgmli_backend.h``; ``backend.Solver`` is its Python binding.
"""
from . import abi  # noqa: F401
