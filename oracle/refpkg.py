"""The installed reference package (mlx-learn 0.1.7) -- TEST INFRASTRUCTURE ONLY.

Only ``tests/`` and ``bench.py``'s reference arm and CPU-baseline legs use
this module, as the checker and as the timed CPU baseline.  The product
(``mlxlearn_b200``) never imports it.

``make -C oracle refpkg`` installs the reference with pip (offline, no
dependencies: MLX does not install here) into ``baseline/_ref`` and places its
two CPU extensions, compiled from the reference's own sources with its own
flags (``make -C oracle ref``), beside its ``_kernels`` package: on Linux the
reference's ``setup.py`` builds no extension, and without them its CPU path
would fall back to NumPy-only engines.  ``baseline/_ref`` travels with the
working tree, so the reference's stock estimators run wherever this
repository does, without the reference source tree.
"""
from __future__ import annotations

import os
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INSTALL = os.path.join(REPO, "baseline", "_ref")


def available() -> bool:
    return os.path.isdir(os.path.join(INSTALL, "mlxlearn"))


def import_reference():
    """The reference's ``mlxlearn`` package with its native CPU engines, or
    None when it is not installed.  Raises if it is installed without them."""
    if not available():
        return None
    if INSTALL not in sys.path:
        sys.path.insert(0, INSTALL)
    import mlxlearn
    import mlxlearn.neighbors  # noqa: F401
    from mlxlearn._kernels import neighbors_cpu, radius_cpu

    if neighbors_cpu._native_query is None or not radius_cpu.AVAILABLE:
        raise RuntimeError("the installed reference lacks its native CPU engines "
                           "(run make -C oracle refpkg)")
    return mlxlearn
