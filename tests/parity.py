"""Comparison helpers of the parity tests.

Tolerance: the target of 1e-10 relative error per step.  Each output field
is compared column by column in the max norm: for field f and column c,
max_g |gpu - ref| <= RTOL * max_g |ref| (plus ATOL for fields that are
identically zero).  Strictly positive fields (densities, temperature) are
also compared element by element: |gpu - ref| <= RTOL * |ref|.
"""
import numpy as np

RTOL = 1e-10
POSITIVE = ("ndensity_s", "rho", "temperature", "ndensity")


def field_errors(gpu: np.ndarray, ref: np.ndarray):
    g = np.asarray(gpu, dtype=np.float64)
    r = np.asarray(ref, dtype=np.float64)
    d = np.abs(g - r)
    scale = np.max(np.abs(r), axis=-2, keepdims=True)  # over cells, per field and column
    norm = np.max(d / np.maximum(scale, 1e-300), axis=-2)
    return float(np.max(norm)), float(np.max(d))


def assert_state_close(gpu: dict, ref: dict, names, rtol: float = RTOL, atol: float = 1e-300):
    report = {}
    for k in names:
        g, r = gpu[k], ref[k]
        assert g.shape == r.shape, (k, g.shape, r.shape)
        assert np.all(np.isfinite(g) == np.isfinite(r)), f"{k}: finite mask differs"
        fin = np.isfinite(r)
        gg, rr = np.where(fin, g, 0.0), np.where(fin, r, 0.0)
        norm, absmax = field_errors(gg, rr)
        report[k] = norm
        assert norm <= rtol or absmax <= atol, f"{k}: normwise rel err {norm:.3e} > {rtol:.1e}"
        if k in POSITIVE:
            rel = np.max(np.abs(gg - rr) / np.maximum(np.abs(rr), 1e-300))
            assert rel <= rtol, f"{k}: elementwise rel err {rel:.3e} > {rtol:.1e}"
    return report
