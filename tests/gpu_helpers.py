"""Shared helpers of the GPU parity tests (compare the CUDA core with the oracle)."""
import numpy as np


def rel_close(a, b, rtol, atol=0.0):
    """Elementwise |a - b| <= rtol * max(|a|, |b|) + atol (NaN == NaN)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    both_nan = np.isnan(a) & np.isnan(b)
    ok = np.abs(a - b) <= rtol * np.maximum(np.abs(a), np.abs(b)) + atol
    return ok | both_nan


def bsdf_records(n, seed, lower_frac=0.2):
    """Config-2 style records: wi on the hemisphere (some below the horizon),
    u2 in [0,1)^2, u1 in [0,1), wo cosine-distributed (some below)."""
    rng = np.random.default_rng(seed)
    z = rng.uniform(-lower_frac, 1, n)
    ph = rng.uniform(0, 2 * np.pi, n)
    s = np.sqrt(1 - z * z)
    wi = np.stack([s * np.cos(ph), s * np.sin(ph), z], 1).astype(np.float32)
    u2 = rng.random((n, 2), dtype=np.float32)
    u1 = rng.random(n, dtype=np.float32)
    z2 = np.sqrt(rng.random(n))
    ph2 = rng.uniform(0, 2 * np.pi, n)
    s2 = np.sqrt(1 - z2 * z2)
    sign = np.where(rng.random(n) < 1 - lower_frac, 1, -1)
    wo = np.stack([s2 * np.cos(ph2), s2 * np.sin(ph2), z2 * sign], 1).astype(np.float32)
    return wi, u2, u1, wo
