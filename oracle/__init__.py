"""CPU oracle for exact neighbour search -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of
``bench.py`` may import this package, and only as the checker.  The product
(``mlxlearn_b200``) never imports, links or executes anything here.

``liboracle.so`` (built from ``knn_oracle.c`` by ``oracle/Makefile``) restates
the results contract of mlxlearn's neighbour path:

* ``knn``: rows ordered by exact squared distance of the float32 coordinates,
  ties by smaller training index (reference
  ``src/mlxlearn/_kernels/_neighbors_cpu_native.cpp:170-190``); distances are
  ``sqrt`` of the canonical float64 sum (``_radius_common.h:348-358``).
* ``radius``: exact membership ``S <= fl64(r*r)`` with CSR rows in ascending
  index order or ``(distance, index)`` order
  (``src/mlxlearn/_kernels/radius_contract.py:1-25``,
  ``radius_result.py:160-187``).

Parity of the oracle itself is pinned in ``tests/test_oracle.py`` against the
reference's own CPU outputs (fixtures in ``tests/golden``) and its known-answer
tests.

``ref_native()`` loads the reference's own compiled CPU extensions from
``oracle/_ref`` (built from the reference sources by ``make -C oracle ref``);
they are used as the timed CPU baseline and as a second checker.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")


def reference_tree() -> str:
    """Where the reference source tree is read from when it is present
    (``MLXLEARN_REFERENCE``; the same variable the Makefile and the fixture
    generator read)."""
    return os.environ.get("MLXLEARN_REFERENCE", "/root/reference")


def build() -> None:
    """Compile liboracle.so and, when the reference tree exists, oracle/_ref
    and the installed reference package (``make -C oracle refpkg``)."""
    subprocess.check_call(["make", "-s", "-C", _HERE, f"PY={sys.executable}"])
    ref = reference_tree()
    if os.path.isdir(os.path.join(ref, "src")):
        subprocess.check_call(["make", "-s", "-C", _HERE, "refpkg", f"PY={sys.executable}",
                               f"REF={ref}"])


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        c_i64, c_int, c_dbl = ctypes.c_int64, ctypes.c_int, ctypes.c_double
        L.orc_knn.argtypes = [_f32p, c_i64, c_i64, _f32p, c_i64, c_i64, c_int, c_i64,
                              ctypes.c_void_p, _i64p, c_int]
        L.orc_knn.restype = c_int
        L.orc_exact_compare.argtypes = [_f32p, _f32p, _f32p, c_i64]
        L.orc_exact_compare.restype = c_int
        L.orc_exact_key.argtypes = [_f32p, _f32p, c_i64, _u64p]
        L.orc_exact_key.restype = None
        L.orc_canonical_d2.argtypes = [_f32p, _f32p, c_i64, c_i64, _f64p]
        L.orc_canonical_d2.restype = None
        L.orc_radius_count.argtypes = [_f32p, c_i64, c_i64, _f32p, c_i64, c_dbl, c_int, c_i64,
                                       _i64p, c_int]
        L.orc_radius_count.restype = c_int
        L.orc_radius_fill.argtypes = [_f32p, c_i64, c_i64, _f32p, c_i64, c_dbl, c_int, c_i64,
                                      _i64p, _i64p, ctypes.c_void_p, c_int, c_int]
        L.orc_radius_fill.restype = c_int
        L.orc_exact_le.argtypes = [_f32p, _f32p, c_i64, c_dbl]
        L.orc_exact_le.restype = c_int
        _LIB = L
    return _LIB


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _threads(nthreads):
    return int(nthreads or os.cpu_count() or 1)


def knn(X, Q, k, *, exclude_self=False, q_offset=0, return_distance=True, nthreads=None):
    """Exact kNN: (float64 distances | None, int64 indices), shape (m, k)."""
    X, Q = _f32(X), _f32(Q)
    m = Q.shape[0]
    idx = np.empty((m, k), np.int64)
    dist = np.empty((m, k), np.float64) if return_distance else None
    rc = lib().orc_knn(X, X.shape[0], X.shape[1], Q, m, int(k), int(bool(exclude_self)),
                       int(q_offset), None if dist is None else dist.ctypes.data, idx,
                       _threads(nthreads))
    if rc:
        raise ValueError("oracle: invalid kNN arguments")
    return dist, idx


def radius(X, Q, r, *, exclude_self=False, q_offset=0, sort_results=False, nthreads=None):
    """Exact radius search as CSR: (indptr int64[m+1], indices int64, distances float64)."""
    X, Q = _f32(X), _f32(Q)
    m = Q.shape[0]
    R2 = float(r) * float(r)
    counts = np.empty(m, np.int64)
    nt = _threads(nthreads)
    if lib().orc_radius_count(X, X.shape[0], X.shape[1], Q, m, R2, int(bool(exclude_self)),
                              int(q_offset), counts, nt):
        raise ValueError("oracle: invalid radius arguments")
    indptr = np.zeros(m + 1, np.int64)
    np.cumsum(counts, out=indptr[1:])
    nnz = int(indptr[-1])
    indices = np.empty(nnz, np.int64)
    dist = np.empty(nnz, np.float64)
    lib().orc_radius_fill(X, X.shape[0], X.shape[1], Q, m, R2, int(bool(exclude_self)),
                          int(q_offset), indptr, indices, dist.ctypes.data,
                          int(bool(sort_results)), nt)
    return indptr, indices, dist


def exact_compare(q, a, b):
    """Exact sign of S(q,a) - S(q,b)."""
    q, a, b = _f32(q), _f32(a), _f32(b)
    return int(lib().orc_exact_compare(q, a, b, q.shape[0]))


def exact_key(q, x):
    """S(q,x) * 2**298 as a Python int (exact)."""
    q, x = _f32(q), _f32(x)
    out = np.zeros(10, np.uint64)
    lib().orc_exact_key(q, x, q.shape[0], out)
    return sum(int(v) << (64 * i) for i, v in enumerate(out))


def exact_le(q, x, R2):
    q, x = _f32(q), _f32(x)
    return bool(lib().orc_exact_le(q, x, q.shape[0], float(R2)))


def canonical_d2(q, X):
    q, X = _f32(q), _f32(X)
    out = np.empty(X.shape[0], np.float64)
    lib().orc_canonical_d2(q, X, X.shape[1], X.shape[0], out)
    return out


def ref_native():
    """The reference's own compiled CPU extensions (oracle/_ref), or None."""
    path = os.path.join(_HERE, "_ref")
    if not os.path.isdir(path):
        return None
    if path not in sys.path:
        sys.path.insert(0, path)
    try:
        import _neighbors_cpu_native  # noqa: F401
        import _radius_cpu_native  # noqa: F401
    except ImportError:
        return None
    import types

    return types.SimpleNamespace(neighbors=sys.modules["_neighbors_cpu_native"],
                                 radius=sys.modules["_radius_cpu_native"])
