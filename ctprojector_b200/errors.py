"""Error reporting of the projector calls.

The reference wrappers print a non-zero status and return the (zero) output
array (e.g. ct_projector/projector/cupy/fan_equiangular.py:186-189).  Here a
non-zero status raises ``CTProjectorError`` by default; ``set_strict(False)``
restores the reference behaviour of printing the status and returning.
"""
from __future__ import annotations

import threading

_state = threading.local()
_default_strict = True


class CTProjectorError(RuntimeError):
    """A projector call failed.  ``code`` is the CUDA runtime code or a CTP_ERR_* code."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = int(code)


def set_strict(strict: bool, *, thread_local: bool = False) -> None:
    """Raise on errors (True, default) or print the status like the reference (False)."""
    global _default_strict
    if thread_local:
        _state.strict = bool(strict)
    else:
        _default_strict = bool(strict)


def is_strict() -> bool:
    return getattr(_state, "strict", _default_strict)
