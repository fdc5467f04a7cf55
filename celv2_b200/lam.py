"""The rate weight ``lambda_q8(qindex)`` the decision rules charge per bit.

In the reference encoder ``lambda_q8`` (src/core/quant.cpp:31-39) is
``llround(0.002 * q^2 * (q120 / q)^0.8 * 256)`` with ``q`` = AVM v1.0.0's AC quantizer step
(``av2_ac_quant_QTX(qindex, 0, 0, AVM_BITS_8) / 8``). AVM is not available here, so the step is
replaced by a labelled, clearly synthetic stand-in, ``1 + qindex / 8``; the real table must be
generated where AVM v1.0.0 is built and passed in with ``set_table``. Every engine (the CUDA
engine, the oracle and the reference CPU engine in the tests) receives the same value for a
qindex, so engine-to-engine parity does not depend on it.
"""
from __future__ import annotations

import math

__all__ = ["standin_table", "lambda_q8", "set_table", "table"]


def _standin(qindex: int) -> int:
    step = 1.0 + qindex / 8.0
    pivot = 1.0 + 120 / 8.0
    v = 0.002 * step * step * (pivot / step) ** 0.8 * 256.0
    return int(math.floor(v + 0.5))


def standin_table() -> list[int]:
    return [_standin(q) for q in range(256)]


_table = standin_table()


def set_table(values) -> None:
    """Replace the table (256 int64 values, e.g. generated from AVM v1.0.0)."""
    vals = [int(v) for v in values]
    if len(vals) != 256:
        raise ValueError("lambda table needs 256 entries")
    _table[:] = vals


def table() -> list[int]:
    return list(_table)


def lambda_q8(qindex: int) -> int:
    return _table[max(0, min(255, int(qindex)))]
