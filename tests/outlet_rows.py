"""Comparison of an outlet record with the reference runner's (steps/_runner.py:104-121)."""
import numpy as np


def same_row(row, ref, rtol, atol=0.0):
    assert set(row) == set(ref), set(row) ^ set(ref)
    for k, v in ref.items():
        a = row[k]
        a = a.value if hasattr(a, "value") else a
        if isinstance(v, str):
            assert a == v, (k, a, v)
        elif v is None or (isinstance(v, float) and np.isnan(v)):
            assert a is None or np.isnan(a), (k, a, v)
        else:
            assert abs(a - v) <= rtol * abs(v) + atol, (k, a, v)
