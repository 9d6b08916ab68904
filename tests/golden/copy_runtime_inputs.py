"""Copy the reference's order-4 runtime inputs (DIR4IN01 files of the
``inputs/runtime/n*`` ladder: 512^2, dk = 0.1, g = h = 1, 50..1500 modes)
into ``tests/golden/runtime/``.  These are the inputs behind the reference's
published eta44 GL / WIT timings (``paper/order4/data/runtime/*.csv``); the
bench's order-4 workload reads the copies, since the reference checkout does
not exist where the bench runs.

Usage: python tests/golden/copy_runtime_inputs.py /path/to/reference (or set GL_REFERENCE)
"""

import os
import shutil
import sys
from pathlib import Path

where = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GL_REFERENCE")
if not where:
    sys.exit("usage: copy_runtime_inputs.py REFERENCE_CHECKOUT (or set GL_REFERENCE)")
src = Path(where) / "paper/order4/inputs/runtime"
dst = Path(__file__).resolve().parent / "runtime"
dst.mkdir(exist_ok=True)
for d in sorted(src.glob("n*")):
    f = d / "directional_eta44_input.bin"
    if f.exists():
        shutil.copy(f, dst / f"{d.name}.bin")
        print(dst / f"{d.name}.bin")
