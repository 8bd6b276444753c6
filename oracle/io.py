"""CPU restatement of the reference's .dat text writers (test infrastructure only).

The checker for ``ss_format_text`` and ``soliton_solver_b200.core.io``; the library never
imports it.  It restates soliton_solver/core/io.py:16-240 as functions returning the
bytes the reference writes: each value as Python's ``format(float(v), ".{p}g")`` and a
tab, a newline after each lattice row (``output_field_dat`` :44-86,
``output_density_data_dat`` :113-151), a blank line after each field component
(``output_field_dat``), no newline at all in ``output_iteration_data_dat`` (:88-111).
Pinned to files the reference wrote (``tests/golden/dat``,
``tests/golden/make_golden_dat.py``).
"""
from __future__ import annotations

import numpy as np


def _fmt(v, precision):
    return f"{{:.{precision}g}}".format(float(v))


def field_text(field_flat, xlen, ylen, nfields, precision=32) -> bytes:
    f = np.asarray(field_flat).reshape(-1)
    parts = []
    for a in range(nfields):
        for x in range(xlen):
            for y in range(ylen):
                parts.append(_fmt(f[y + x * ylen + a * xlen * ylen], precision))
                parts.append("\t")
            parts.append("\n")
        parts.append("\n")
    return "".join(parts).encode()


def density_text(density_flat, a, xlen, ylen, precision=32) -> bytes:
    d = np.asarray(density_flat).reshape(-1)
    parts = []
    for x in range(xlen):
        for y in range(ylen):
            parts.append(_fmt(d[y + x * ylen + a * xlen * ylen], precision))
            parts.append("\t")
        parts.append("\n")
    return "".join(parts).encode()


def iteration_text(values, precision=32) -> bytes:
    return "".join(_fmt(v, precision) + "\t" for v in values).encode()
