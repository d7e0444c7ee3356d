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


def min_sin_theta(oracle, scene, cam):
    """Per pixel, the smallest sin(theta) its camera ray's geodesic can reach:
    from the constants of motion at the camera (E = -k_t, L_z = k_phi and the
    Carter constant Q = k_theta^2 + cos^2 theta (L_z^2 / sin^2 theta - a^2 E^2)),
    the turning point of the theta motion, sin^2 theta_min ~ L_z^2 / (Q + a^2 E^2
    + L_z^2). Rays with a small value pass close to the spin axis, where
    Boyer-Lindquist coordinates are ill-conditioned."""
    rays = oracle.camera_rays(scene, cam)
    g = oracle.metric(scene, rays[0, :4])
    k = rays[:, 4:8] @ g.T  # lower-index momenta (g is symmetric)
    E, Lz, kth = -k[:, 0], k[:, 3], k[:, 2]
    th = rays[0, 2]
    a = scene.spin if scene.kind in (2, 3, 4, 5) else 0.0
    Q = kth ** 2 + np.cos(th) ** 2 * (Lz ** 2 / np.sin(th) ** 2 - a * a * E ** 2)
    return np.sqrt(Lz ** 2 / np.maximum(Q + a * a * E ** 2 + Lz ** 2, 1e-300))
