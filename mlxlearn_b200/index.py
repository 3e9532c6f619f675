"""The drop-in seam: ``NeighborIndex`` / ``build_index`` on the CUDA library.

Mirrors ``mlxlearn._kernels.distance.NeighborIndex`` (reference
src/mlxlearn/_kernels/distance.py:66-392): the estimators call only
``build_index`` and the index methods below, and get back float64 distances
and int64 indices in ``(distance, index)`` order.  Every query runs on the
GPU through libb200knn.so; there is no CPU route.
"""
from __future__ import annotations

import ctypes
import threading

import numpy as np

from . import _lib

__all__ = ["NeighborIndex", "build_index"]

NUMPY_FLOAT = np.float32
INDEX_DTYPE = np.int64

# Route names of the reference's query policy (src/mlxlearn/_kernels/
# distance.py:114-141): "cpu" asks the calling estimator to take results as
# host arrays through query(), "mlx" to keep them on the device through
# query_device() and vote with MLX.  This index answers every route on the
# GPU; it names the host-array route, the one an estimator can consume
# without MLX (reference src/mlxlearn/neighbors/_classification.py:138-159).
HOST_ARRAY_ROUTE = "cpu"


def _as_f32_c(X) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(X, dtype=NUMPY_FLOAT))


class NeighborIndex:
    """Owned training rows plus a device-resident search index.

    The host float32 copy serves pickling and ``training_data``; the device
    copy (created lazily on first use, or eagerly by ``build_index``) is the
    only thing searched.
    """

    def __init__(self, X: np.ndarray, *, device: int = 0, mode: str = "auto",
                 backend: str = "cuda", auto_policy: bool = False):
        if X.ndim != 2 or 0 in X.shape:
            raise ValueError("X must be a nonempty two-dimensional matrix")
        if X.shape[0] >= 2**31:
            raise ValueError("training row count must fit int32 indices")
        self._host_X = X
        self._n, self._d = int(X.shape[0]), int(X.shape[1])
        self.device = int(device)
        self.mode = mode
        # the backend name and policy flag the estimator asked for at fit
        # (reference distance.py:86-97); every query runs on the GPU anyway
        self.backend = backend
        self.auto_policy = bool(auto_policy)
        self._gpu_available = True
        self._handle = None
        self._lock = threading.Lock()
        self.last_query_backend = None
        self.last_stats = None

    @classmethod
    def from_device(cls, X, *, mode: str = "auto") -> "NeighborIndex":
        """Index over a CUDA float32 tensor ``[n, d]`` (copied on the current
        stream; no host round trip).  ``training_data`` is downloaded lazily."""
        import torch

        if not (isinstance(X, torch.Tensor) and X.is_cuda and X.dim() == 2):
            raise TypeError("from_device expects a 2-D CUDA tensor")
        if 0 in X.shape:
            raise ValueError("X must be a nonempty two-dimensional matrix")
        Xc = X.detach().to(torch.float32).contiguous()
        self = cls.__new__(cls)
        self._host_X = None
        self._n, self._d = int(Xc.shape[0]), int(Xc.shape[1])
        self.device = Xc.device.index or 0
        self.mode = mode
        self.backend = "cuda"
        self.auto_policy = False
        self._gpu_available = True
        self._lock = threading.Lock()
        self.last_query_backend = None
        self.last_stats = None
        lib = _lib.load()
        h = ctypes.c_void_p()
        stream = torch.cuda.current_stream(Xc.device).cuda_stream
        _lib.check(lib.b2k_index_create_device(Xc.data_ptr(), self._n, self._d, stream,
                                               ctypes.byref(h)), "b2k_index_create_device")
        self._handle = h
        return self

    # ------------------------------------------------------------ lifetime
    def _ensure_device(self):
        if self._handle is None:
            with self._lock:
                if self._handle is None:
                    lib = _lib.load()
                    h = ctypes.c_void_p()
                    X = self._host_X
                    _lib.check(lib.b2k_index_create(X.ctypes.data, X.shape[0], X.shape[1],
                                                    self.device, ctypes.byref(h)),
                               "b2k_index_create")
                    self._handle = h
        return self._handle

    def close(self):
        if self._handle is not None and _lib._lib is not None:
            _lib._lib.b2k_index_destroy(self._handle)
        self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __getstate__(self):
        # Host rows and parameters only; the device index is rebuilt lazily
        # (reference distance.py:191-209).
        return {"X": self.training_data, "device": self.device, "mode": self.mode,
                "backend": self.backend, "auto_policy": self.auto_policy}

    def __setstate__(self, state):
        self.__init__(state["X"], device=state.get("device", 0), mode=state.get("mode", "auto"),
                      backend=state.get("backend", "cuda"),
                      auto_policy=state.get("auto_policy", False))

    @property
    def device_index(self) -> "NeighborIndex":
        """The device-resident search state (reference distance.py:179-182):
        this object, with its library index created."""
        self._ensure_device()
        return self

    # ----------------------------------------------------------- properties
    @property
    def training_data(self) -> np.ndarray:
        if self._host_X is None:
            X = np.empty((self._n, self._d), dtype=NUMPY_FLOAT)
            _lib.check(_lib.load().b2k_index_download(self._handle, X.ctypes.data),
                       "b2k_index_download")
            self._host_X = X
        return self._host_X

    @property
    def X(self) -> np.ndarray:
        return self.training_data

    @property
    def n_samples(self) -> int:
        return self._n

    @property
    def n_features(self) -> int:
        return self._d

    # -------------------------------------------------------------- queries
    def _query_policy(self, n_query, k, Q=None):
        """``(route, integer_exact)`` as the reference's policy returns it
        (distance.py:114-138).  Every batch runs on the GPU; the route is the
        host-array one (``HOST_ARRAY_ROUTE``) and no integer-exact variant
        is needed because every answer is exact."""
        return HOST_ARRAY_ROUTE, None

    def backend_for_query(self, n_query, k, Q=None):
        return self._query_policy(n_query, k, Q)[0]

    def _check_query(self, n_query: int, k: int, exclude_self: bool):
        limit = self.n_samples - int(bool(exclude_self))
        if k > limit:
            raise ValueError(f"n_neighbors must be <= {limit}, got {k}.")
        if exclude_self and n_query != self.n_samples:
            raise ValueError(
                "exclude_self requires the query matrix to be the training matrix: "
                f"got {n_query} query rows and {self.n_samples} training rows.")

    def query(self, Q, k, *, return_distance=True, exclude_self=False,
              query_block_size=None, train_block_size=None, _policy=None, mode=None,
              stats=False, out=None):
        """Float64 distances (or None) and int64 indices, each ``[n_query, k]``.

        ``query_block_size`` splits the queries into independent batches;
        results do not depend on it.  ``train_block_size`` is accepted for
        compatibility: the engine tiles the training rows itself and its
        merge is exact, so blocking never changes an answer.  ``_policy``
        (a ``_query_policy`` result, reference distance.py:242-245) does not
        change the route: every policy runs here.  ``out`` may supply
        preallocated (e.g. pinned) ``(dist, idx)`` host arrays.
        """
        Q = _as_f32_c(Q)
        k = int(k)
        if Q.ndim != 2 or Q.shape[1] != self.n_features:
            raise ValueError(f"Q must have shape (n, {self.n_features})")
        m = Q.shape[0]
        self._check_query(m, k, exclude_self)
        if out is not None:
            dist, idx = out
            if idx.shape != (m, k) or idx.dtype != INDEX_DTYPE or not idx.flags.c_contiguous:
                raise ValueError("out indices must be a C-contiguous int64 array of shape (m, k)")
            if dist is not None and (dist.shape != (m, k) or dist.dtype != np.float64
                                     or not dist.flags.c_contiguous):
                raise ValueError("out distances must be a C-contiguous float64 array (m, k)")
            if not return_distance:
                dist = None
        else:
            idx = np.empty((m, k), dtype=INDEX_DTYPE)
            dist = np.empty((m, k), dtype=np.float64) if return_distance else None
        if m:
            h = self._ensure_device()
            lib = _lib.load()
            code = _lib.MODES[mode or self.mode]
            st = _lib.Stats()
            step = m if not query_block_size else max(1, int(query_block_size))
            for start in range(0, m, step):
                stop = min(m, start + step)
                rc = lib.b2k_knn(h, Q[start:stop].ctypes.data, stop - start, k,
                                 int(bool(exclude_self)), start, code,
                                 None if dist is None else dist[start:stop].ctypes.data,
                                 idx[start:stop].ctypes.data, ctypes.byref(st) if stats else None)
                _lib.check(rc, "b2k_knn")
            self.last_stats = st.as_dict() if stats else None
        self.last_query_backend = "cuda"
        return dist, idx

    def query_device(self, Q, k, *, return_distance=True, exclude_self=False,
                     query_block_size=None, train_block_size=None, _squared=False, q_offset=0,
                     mode=None, stats=False, stream=None):
        """Device-resident query (reference distance.py:211-240): ``Q`` is a
        CUDA float32 tensor ``[m, d]`` (a host array is uploaded first).

        Returns torch tensors on the device (float64 distances or None, int64
        indices), computed on the current torch stream.  ``_squared`` returns
        the canonical float64 squared distances instead of their square
        roots.  ``query_block_size`` splits the batch (results do not depend
        on it); ``train_block_size`` is accepted for compatibility.
        """
        import torch

        if not (isinstance(Q, torch.Tensor) and Q.is_cuda):
            if isinstance(Q, torch.Tensor):
                raise TypeError("query_device expects a CUDA tensor or a host array")
            Q = torch.from_numpy(_as_f32_c(Q)).to(torch.device("cuda", self.device))
        Q = Q.detach().to(torch.float32).contiguous()
        m, k = int(Q.shape[0]), int(k)
        if Q.dim() != 2 or (m and Q.shape[1] != self.n_features):
            raise ValueError(f"Q must have shape (n, {self.n_features})")
        if exclude_self:
            limit = self.n_samples - 1
            if k > limit:
                raise ValueError(f"n_neighbors must be <= {limit}, got {k}.")
        elif k > self.n_samples:
            raise ValueError(f"n_neighbors must be <= {self.n_samples}, got {k}.")
        idx = torch.empty((m, k), dtype=torch.int64, device=Q.device)
        dist = torch.empty((m, k), dtype=torch.float64, device=Q.device) if return_distance else None
        if m:
            h = self._ensure_device()
            st = _lib.Stats()
            s = stream if stream is not None else torch.cuda.current_stream(Q.device).cuda_stream
            code = _lib.MODES[mode or self.mode] | (_lib.MODE_SQUARED if _squared else 0)
            step = m if not query_block_size else max(1, int(query_block_size))
            for start in range(0, m, step):
                stop = min(m, start + step)
                rc = _lib.load().b2k_knn_device(
                    h, Q[start:stop].data_ptr(), stop - start, k, int(bool(exclude_self)),
                    int(q_offset) + start, code,
                    None if dist is None else dist[start:stop].data_ptr(),
                    idx[start:stop].data_ptr(), s, ctypes.byref(st) if stats else None)
                _lib.check(rc, "b2k_knn_device")
            self.last_stats = st.as_dict() if stats else None
        self.last_query_backend = "cuda"
        return dist, idx


    # ----------------------------------------------------------------- radius
    def query_radius_csr(self, Q, radius, *, need_distance=True, exclude_self=False,
                         sort_results=False, algorithm="auto", n_jobs=None, patched=False,
                         query_block_size=None, raw=False):
        """Neighbourhoods within an inclusive Euclidean radius, as CSR batches.

        A training row is returned iff its exact squared distance is at most
        ``fl64(radius ** 2)`` (reference distance.py:285-342).  Rows hold
        ascending training indices, or ``(distance, index)`` order with
        ``sort_results``.  With ``raw`` each batch keeps its device result,
        so ``votes``/``mean`` reduce it on the GPU and host arrays are only
        copied if read; otherwise the batches are copied into page-locked
        host memory at once and the device results freed.
        ``algorithm``/``n_jobs``/``patched`` are accepted for signature
        compatibility.
        """
        from .radius_result import RadiusCSR

        radius = validate_radius(radius)
        Q = _as_f32_c(Q)
        if Q.ndim != 2 or Q.shape[1] != self.n_features:
            raise ValueError(f"Q must have shape (n, {self.n_features})")
        n_query = int(Q.shape[0])
        if exclude_self and n_query != self.n_samples:
            raise ValueError(
                "exclude_self requires the query matrix to be the training matrix: "
                f"got {n_query} query rows and {self.n_samples} training rows.")
        step = n_query if not query_block_size else max(1, int(query_block_size))
        parts = []
        lib = _lib.load()
        h = self._ensure_device()
        for start in range(0, max(n_query, 1), max(step, 1)):
            stop = min(n_query, start + step)
            block = Q[start:stop]
            res = ctypes.c_void_p()
            rc = lib.b2k_radius(h, block.ctypes.data if len(block) else None, stop - start,
                                float(radius), int(bool(exclude_self)), start,
                                int(bool(need_distance or sort_results)),
                                int(bool(sort_results)), ctypes.byref(res))
            _lib.check(rc, "b2k_radius")
            part = RadiusCSR.from_device(res, stop - start, device=self.device,
                                         distances=bool(need_distance))
            if not raw:
                part.indptr  # noqa: B018 -- copy out now, then free the device result
                part.release()
            parts.append(part)
        self.last_query_backend = "cuda"
        return parts

    def query_radius_reduce(self, Q, radius, *, codes=None, n_classes=0, targets=None,
                            weighted=False, exclude_self=False, query_block_size=None):
        """Per-query class votes (``codes``: CUDA int32 labels of the training
        rows) or target means (``targets``: CUDA float64) over the radius
        neighbourhoods, reduced on the device without downloading them.
        Returns ``(votes [m, n_classes] or means [m], counts [m])`` as numpy
        arrays, equal to the host reductions over :meth:`query_radius_csr`."""
        if (codes is None) == (targets is None):
            raise ValueError("pass exactly one of codes and targets")
        parts = self.query_radius_csr(Q, radius, need_distance=bool(weighted),
                                      exclude_self=exclude_self,
                                      query_block_size=query_block_size, raw=True)
        pieces = [p.votes(codes, n_classes, weighted) if codes is not None
                  else p.mean(targets, weighted) for p in parts]
        for p in parts:
            p.release()
        if len(pieces) == 1:
            return pieces[0]
        return (np.concatenate([a for a, _ in pieces]), np.concatenate([c for _, c in pieces]))

    def query_radius_predict(self, Q, radius, *, codes, n_classes, exclude_self=False,
                             query_block_size=None):
        """Per-query first maximum of the class counts within ``radius``
        (uniform weights; ties -> smallest code, 0 for an empty row) and the
        counts, as numpy int64 arrays: the argmax of the normalised votes,
        computed on the device without downloading the votes."""
        parts = self.query_radius_csr(Q, radius, need_distance=False, exclude_self=exclude_self,
                                      query_block_size=query_block_size, raw=True)
        pieces = [p.predict_codes(codes, n_classes) for p in parts]
        for p in parts:
            p.release()
        if len(pieces) == 1:
            return pieces[0]
        return (np.concatenate([a for a, _ in pieces]), np.concatenate([c for _, c in pieces]))

    def query_radius(self, Q, radius, *, return_distance=True, exclude_self=False,
                     sort_results=False, query_block_size=None, train_block_size=None,
                     algorithm="auto"):
        """scikit-learn's ragged form of :meth:`query_radius_csr`."""
        from .radius_result import ragged_rows

        if Q.shape[0] == 0:
            empty = np.empty(0, dtype=object)
            return (np.empty(0, dtype=object), empty) if return_distance else empty
        parts = self.query_radius_csr(Q, radius, need_distance=return_distance or sort_results,
                                      exclude_self=exclude_self, sort_results=sort_results,
                                      query_block_size=query_block_size)
        return ragged_rows(parts, return_distance=return_distance)


def validate_radius(radius) -> float:
    """A radius as a float; rejects NaN, negatives, booleans and arrays
    (reference src/mlxlearn/_kernels/radius_contract.py:75-95)."""
    import math
    from numbers import Real

    if isinstance(radius, np.ndarray):
        if radius.ndim != 0:
            raise TypeError(f"radius must be a scalar, got an array of shape {radius.shape}")
        radius = radius[()]
    if isinstance(radius, (bool, np.bool_)) or not isinstance(radius, (Real, np.floating,
                                                                        np.integer)):
        raise TypeError(f"radius must be a real number, got {type(radius).__name__}")
    value = float(radius)
    if math.isnan(value):
        raise ValueError("radius must not be NaN")
    if value < 0:
        raise ValueError(f"radius must be non-negative, got {value}")
    return value + 0.0


def build_index(X, *, backend: str = "cuda", _owned: bool = False, _auto: bool = False,
                _gpu_available=True, device: int = 0, mode: str = "auto") -> NeighborIndex:
    """Own a float32 C-order copy of ``X`` (never alias a caller's array).

    Takes the reference's arguments (distance.py:366-392): ``backend`` and
    ``_auto`` are recorded on the index, ``_gpu_available`` is accepted;
    every backend name runs on the CUDA library.  ``_owned`` hands over a
    freshly converted buffer instead of copying it.
    """
    Xf = (np.ascontiguousarray(np.asarray(X, dtype=NUMPY_FLOAT)) if _owned
          else np.array(X, dtype=NUMPY_FLOAT, order="C", copy=True))
    return NeighborIndex(Xf, device=device, mode=mode, backend=backend, auto_policy=_auto)
