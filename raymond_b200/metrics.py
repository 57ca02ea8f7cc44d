"""Image error metrics against a converged reference."""
from __future__ import annotations

import numpy as np


def relmse(image: np.ndarray, reference: np.ndarray, eps: float = 1e-2) -> float:
    """Relative mean squared error: mean over pixels and channels of
    (x - ref)^2 / (lum(ref)^2 + eps), with the mean over channels of ref as the
    pixel's luminance proxy (Rousselle et al. 2011)."""
    x = np.asarray(image, np.float64)
    ref = np.asarray(reference, np.float64)
    lum = ref.mean(axis=-1, keepdims=True)
    return float(np.mean((x - ref) ** 2 / (lum * lum + eps)))
