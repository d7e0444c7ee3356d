"""Parity metrics between the CUDA library and the oracle (test helpers)."""
import numpy as np


def class_match(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.mean(a == b)) if a.size else 1.0


def rel_err(gpu, ref, floor_frac=1e-6):
    """Per-pixel relative error with denominator max(|ref|, floor_frac * max|ref|)."""
    gpu = np.asarray(gpu, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    scale = np.max(np.abs(ref)) if ref.size else 0.0
    den = np.maximum(np.abs(ref), floor_frac * scale + 1e-300)
    return np.abs(gpu - ref) / den


def summarize(gpu, ref, mask=None):
    """Fraction of pixels within 1e-3 relative error on linear XYZ (Y), over the
    pixels whose termination class agrees (and `mask`)."""
    same = np.asarray(gpu["class"]) == np.asarray(ref["class"])
    if mask is not None:
        same &= mask
    e = rel_err(gpu["xyz"][:, 1], ref["xyz"][:, 1])[same]
    return {
        "class_match": class_match(gpu["class"], ref["class"]),
        "n": int(same.sum()),
        "frac_within_1e-3": float(np.mean(e <= 1e-3)) if e.size else 1.0,
        "max_rel": float(e.max()) if e.size else 0.0,
        "p99_rel": float(np.quantile(e, 0.99)) if e.size else 0.0,
    }
