"""B200-native implementation of AndoSim's implicit cloth/shell step.

``andosim_b200.ando_barrier_core`` is the drop-in for the reference's
``ando_barrier_core`` pybind11 module; it runs the step on the GPU through the
C ABI in ``include/ando_gpu.h`` (``andosim_b200/lib/libando_gpu.so``).
The extension is built in-tree by ``andosim_b200.build.build()``; importing this
package never falls back to a CPU implementation.
"""
from __future__ import annotations

from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent
GPU_LIBRARY = PACKAGE_DIR / "lib" / "libando_gpu.so"


def load_core():
    """Import and return the ``ando_barrier_core`` extension module."""
    from . import ando_barrier_core  # noqa: F401  (raises ImportError when not built)

    return ando_barrier_core
