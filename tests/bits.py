"""Bit-level equality for parity tests.

``numpy.testing.assert_array_equal`` compares values, so -0.0 equals +0.0 and
NaN equals NaN; a bit-exact claim needs the bit patterns compared, which is
what ``assert_bits_equal`` does (same dtype and shape, then every byte)."""
import numpy as np


def assert_bits_equal(a, b, err_msg: str = "") -> None:
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    where = f"{err_msg}: " if err_msg else ""
    if a.dtype != b.dtype or a.shape != b.shape:
        raise AssertionError(f"{where}dtype/shape {a.dtype}{a.shape} vs {b.dtype}{b.shape}")
    if a.tobytes() == b.tobytes():
        return
    w = a.dtype.itemsize
    ua = np.frombuffer(a.tobytes(), np.uint8).reshape(-1, w)
    ub = np.frombuffer(b.tobytes(), np.uint8).reshape(-1, w)
    bad = np.flatnonzero(np.any(ua != ub, axis=1))
    q = int(bad[0])
    fa, fb = a.reshape(-1)[q], b.reshape(-1)[q]
    vals_equal = bool(np.all(a.reshape(-1)[bad] == b.reshape(-1)[bad]))
    raise AssertionError(f"{where}{len(bad)} of {a.size} values differ in their bits "
                         f"({'all equal as values: signed zeros or NaN payloads' if vals_equal else 'values differ'}); "
                         f"first at flat index {q}: {fa!r} vs {fb!r}")
