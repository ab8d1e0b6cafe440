"""Build libwake_b200.so in-tree for sm_100a (``python wake_b200/build.py``).

Run as a file (or load by path): importing the wake_b200 package needs the
library this builds."""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def build(jobs: int | None = None, verbose: bool = False) -> Path:
    jobs = jobs or max(1, min(8, os.cpu_count() or 1))
    cmd = ["make", "-C", str(HERE / "csrc"), f"-j{jobs}"]
    out = subprocess.run(cmd, capture_output=not verbose, text=True)
    if out.returncode != 0:
        sys.stderr.write((out.stdout or "") + (out.stderr or ""))
        raise RuntimeError("building libwake_b200.so failed")
    return HERE / "libwake_b200.so"


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
