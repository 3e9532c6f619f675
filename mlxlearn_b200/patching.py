"""Point scikit-learn's neighbour estimators at this package's classes.

The same entry points as the reference's patching shell
(src/mlxlearn/patching/_patch.py:63-255): ``patch_sklearn``,
``unpatch_sklearn``, ``is_patched``, ``get_patch_map`` and
``patched_estimators``, restricted to the five estimators of the
neighbour path.  Behaviour kept from the reference: names resolve bare
(``"KNeighborsClassifier"``) or dotted (``"sklearn.neighbors.KNeighborsClassifier"``);
an unknown name raises ValueError listing what is available, in both
directions; patching is idempotent and records the original class once; a
class that something else installed after us is left alone with a warning.
Patch before importing the names you want accelerated: ``from
sklearn.neighbors import X`` made earlier keeps the class it bound.
"""
from __future__ import annotations

import importlib
import sys
import threading
import warnings
from dataclasses import dataclass

__all__ = ["patch_sklearn", "unpatch_sklearn", "is_patched", "get_patch_map",
           "patched_estimators", "PatchWarning"]


class PatchWarning(UserWarning):
    """A patch or unpatch was skipped to keep another library's replacement."""


@dataclass(frozen=True)
class _Spec:
    attribute: str
    module: str = "sklearn.neighbors"

    @property
    def name(self) -> str:
        return f"{self.module}.{self.attribute}"


_SPECS = [_Spec(a) for a in ("NearestNeighbors", "KNeighborsClassifier", "KNeighborsRegressor",
                             "RadiusNeighborsClassifier", "RadiusNeighborsRegressor")]
_LOOKUP = {**{s.attribute: s for s in _SPECS}, **{s.name: s for s in _SPECS}}
_lock = threading.RLock()
_installed: dict[str, tuple[object, object]] = {}  # name -> (original, ours)


def _resolve(estimators) -> list[_Spec]:
    if estimators is None:
        return list(_SPECS)
    names = [estimators] if isinstance(estimators, str) else list(estimators)
    out: list[_Spec] = []
    for n in names:
        spec = _LOOKUP.get(n)
        if spec is None:
            available = ", ".join(s.attribute for s in _SPECS)
            raise ValueError(f"no accelerated implementation is registered for {n!r}. "
                             f"Available: {available}. Pass estimators=None for all of them.")
        if spec not in out:
            out.append(spec)
    return out


def _ours(spec: _Spec):
    from . import neighbors

    return getattr(neighbors, spec.attribute)


def patch_sklearn(estimators=None, verbose: bool = False) -> None:
    specs = _resolve(estimators)
    with _lock:
        module = importlib.import_module("sklearn.neighbors")
        for spec in specs:
            current = getattr(module, spec.attribute)
            entry = _installed.get(spec.name)
            if entry is not None:
                if current is not entry[1]:
                    warnings.warn(f"{spec.name} was replaced by another object after it was "
                                  "patched; leaving that replacement in place. Call "
                                  "unpatch_sklearn() first to re-patch.", PatchWarning,
                                  stacklevel=2)
                continue
            ours = _ours(spec)
            _installed[spec.name] = (current, ours)
            setattr(module, spec.attribute, ours)
    if verbose and sys.stderr is not None:
        print("mlxlearn_b200: patched scikit-learn estimators [" +
              ", ".join(s.attribute for s in specs) + "]", file=sys.stderr)


def unpatch_sklearn(estimators=None) -> None:
    specs = _resolve(estimators)
    with _lock:
        module = importlib.import_module("sklearn.neighbors")
        for spec in specs:
            entry = _installed.pop(spec.name, None)
            if entry is None:
                continue  # never patched: nothing to restore
            original, ours = entry
            if getattr(module, spec.attribute) is not ours:
                warnings.warn(f"{spec.name} is no longer the class installed here; not "
                              "restoring it, to keep the later replacement.", PatchWarning,
                              stacklevel=2)
                continue
            setattr(module, spec.attribute, original)


def _patched_one(spec: _Spec) -> bool:
    entry = _installed.get(spec.name)
    if entry is None:
        return False
    module = sys.modules.get(spec.module)
    return module is not None and getattr(module, spec.attribute, None) is entry[1]


def is_patched(estimators=None) -> bool:
    with _lock:
        specs = _resolve(estimators)
        return bool(specs) and all(_patched_one(s) for s in specs)


def get_patch_map() -> dict[str, dict[str, object]]:
    with _lock:
        out = {}
        for spec in _SPECS:
            entry = _installed.get(spec.name)
            out[spec.name] = {
                "module": spec.module,
                "attribute": spec.attribute,
                "patched": _patched_one(spec),
                "accelerated_class": f"mlxlearn_b200.neighbors.{spec.attribute}",
                "original": entry[0] if entry else None,
            }
        return out


def patched_estimators() -> list[str]:
    with _lock:
        return [s.name for s in _SPECS if _patched_one(s)]
