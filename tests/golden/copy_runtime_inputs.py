"""Copy the reference's order-4 runtime inputs (DIR4IN01 files of the
``inputs/runtime/n*`` ladder: 512^2, dk = 0.1, g = h = 1, 50..1500 modes)
into ``tests/golden/runtime/``.  These are the inputs behind the reference's
published eta44 GL / WIT timings (``paper/order4/data/runtime/*.csv``); the
bench's order-4 workload reads the copies, since the reference checkout does
not exist where the bench runs.

Usage: python tests/golden/copy_runtime_inputs.py /path/to/reference
"""

import shutil
import sys
from pathlib import Path

src = Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference") / "paper/order4/inputs/runtime"
dst = Path(__file__).resolve().parent / "runtime"
dst.mkdir(exist_ok=True)
for d in sorted(src.glob("n*")):
    f = d / "directional_eta44_input.bin"
    if f.exists():
        shutil.copy(f, dst / f"{d.name}.bin")
        print(dst / f"{d.name}.bin")
