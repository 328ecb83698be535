"""SciPy ``LinearOperator`` adapter (``python/tencirpauli/integrations/scipy.py:13-49``)."""

from __future__ import annotations

from typing import Any, Optional

import numpy as np

from .._native_mvp import DEFAULT_MAX_BYTES, validate_max_bytes


def to_scipy_linear_operator(plan: Any, *, max_bytes: Optional[int] = DEFAULT_MAX_BYTES) -> Any:
    """Wrap one immutable MVP plan as a matrix-free ``LinearOperator``."""
    from scipy.sparse.linalg import LinearOperator

    validate_max_bytes(max_bytes)
    dimension = int(plan.dimension)

    def matvec(vector: Any) -> np.ndarray:
        values = np.asarray(vector, dtype=np.complex128)
        if values.ndim == 2:
            if values.shape != (dimension, 1):
                raise ValueError(
                    f"LinearOperator vector must have shape ({dimension},) or ({dimension}, 1), got {values.shape}"
                )
            values = values[:, 0]
        elif values.ndim != 1 or values.shape != (dimension,):
            raise ValueError(
                f"LinearOperator vector must have shape ({dimension},) or ({dimension}, 1), got {values.shape}"
            )
        return np.asarray(plan.apply(np.ascontiguousarray(values), max_bytes=max_bytes), dtype=np.complex128)

    return LinearOperator(shape=(dimension, dimension), matvec=matvec, dtype=np.complex128)


__all__ = ["to_scipy_linear_operator"]
