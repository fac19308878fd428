"""Per-block layout of the loaded build.

The reference fixes its ghost layers at compile time (PRJ_NGHOST: 2, or 4
when WENO-Z7 is selected, src/prj_defs.h:339-351); so does this package: the
environment variable FX_NGHOST (2 by default, or 4) selects the library
(libfornax_b200.so or libfornax_b200_ng4.so) and every size below, for the
whole process.
"""
from __future__ import annotations

import os

BS = 16
NG = int(os.environ.get("FX_NGHOST", "2"))
if NG not in (2, 4):
    raise ValueError("FX_NGHOST must be 2 or 4")
PBS = BS + 2 * NG
NCELLS = PBS ** 3
NFACES = (PBS + 1) * PBS * PBS
NEDGES = (PBS + 1) * (PBS + 1) * PBS
