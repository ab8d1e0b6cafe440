#!/usr/bin/env python3
"""Build recipe for the reference's own CPU lattice-update path (test infrastructure only).

The reference (Aneesh495/wake) compiles its kernels with the ISPC compiler
(src/ispc/CMakeLists.txt:1-36, target avx2-i32x8, --opt=fast-math). ISPC is not
installed in this image, so the kernel sources are translated mechanically into
C++ at build time:

  * ``foreach (i = a ... b)``   -> ``for (int i = a; i < b; ++i)``
  * ``export``                  -> ``extern "C"``
  * ``uniform`` / ``varying``   -> dropped (one lane per loop iteration)
  * ``uint8``                   -> ``uint8_t``;  ``reduce_add(x)`` -> ``x``

Nothing else is changed: every arithmetic expression is the reference's own.
The translated files are written to ``oracle/_ref/gen`` and compiled with g++
(-O3 -march=x86-64-v3 -ffast-math, mirroring ISPC's avx2 fast-math build; the host
sources with the reference's own C++ flags, -O3 -pthread)
together with the reference's host C++ compiled from where it lies
(src/grid/lattice_grid_2d.cpp, src/grid/lattice_grid_3d.cpp, src/core/memory.cpp,
src/forces/strouhal_analyzer.cpp, src/export/csv_telemetry.cpp, src/export/vtk_exporter.cpp)
and the thin extern "C" shim ``oracle/ref_shim.cpp``. The output is
``oracle/_ref/libwake_ref.so``. Nothing is copied into the repository: the
output directory is git-ignored.

Only tests, the smoke check and bench.py's reference arm use the result.
"""
from __future__ import annotations

import os
import re
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
GEN = OUT / "gen"

PRELUDE_H = """#pragma once
#include <cmath>
#include <cstdint>
#include <algorithm>
using std::sqrt; using std::min; using std::max; using std::floor; using std::abs; using std::cos;
typedef uint8_t uint8;
static inline float reduce_add(float v) { return v; }
"""
PRELUDE = '// Mechanically translated from ISPC by oracle/build_ref.py. Do not edit.\n#include "ispc_prelude.h"\n'


FOREACH = re.compile(r"foreach\s*\(\s*(\w+)\s*=\s*(.+?)\s*\.\.\.\s*(.+?)\s*\)\s*\{")


def reference_dir() -> Path:
    """The reference checkout: WAKE_REFERENCE_DIR, else a directory named `reference` beside
    the one that holds this repository."""
    env = os.environ.get("WAKE_REFERENCE_DIR")
    return Path(env) if env else Path(__file__).resolve().parents[2] / "reference"


def translate(text: str) -> str:
    text = FOREACH.sub(lambda m: f"for (int {m.group(1)} = {m.group(2)}; {m.group(1)} < {m.group(3)}; ++{m.group(1)}) {{", text)
    text = re.sub(r"\bexport\s+void\b", 'extern "C" void', text)
    text = re.sub(r"\b(uniform|varying)\b\s*", "", text)
    return text


def build(verbose: bool = False) -> Path:
    ref = reference_dir()
    if not (ref / "src" / "ispc").is_dir():
        raise FileNotFoundError(f"reference sources not found under {ref}")
    (GEN / "include" / "wake" / "ispc").mkdir(parents=True, exist_ok=True)
    (GEN / "include" / "ispc_prelude.h").write_text(PRELUDE_H)
    for isph in sorted((ref / "include" / "wake" / "ispc").glob("*.isph")):
        body = translate(isph.read_text())
        (GEN / "include" / "wake" / "ispc" / isph.name).write_text(PRELUDE + body)
    cpp_files = []
    for ispc in sorted((ref / "src" / "ispc").glob("*.ispc")):
        dst = GEN / (ispc.stem + ".cpp")
        dst.write_text(PRELUDE + translate(ispc.read_text()))
        cpp_files.append(str(dst))
    host = [ref / "src" / "grid" / "lattice_grid_2d.cpp",
            ref / "src" / "grid" / "lattice_grid_3d.cpp",
            ref / "src" / "core" / "memory.cpp",
            ref / "src" / "forces" / "strouhal_analyzer.cpp",
            ref / "src" / "export" / "csv_telemetry.cpp",
            ref / "src" / "export" / "vtk_exporter.cpp"]
    so = OUT / "libwake_ref.so"
    # the translated kernels with ISPC's fast-math avx2 settings (CMakeLists.txt:24), the
    # host sources with the reference's C++ flags (CMakeLists.txt:25)
    objs = OUT / "obj"
    objs.mkdir(parents=True, exist_ok=True)
    inc = [f"-I{GEN / 'include'}", f"-I{ref / 'include'}"]
    jobs = []
    for src in cpp_files:
        jobs.append(["g++", "-std=c++20", "-O3", "-march=x86-64-v3", "-ffast-math", "-fPIC", *inc, "-c", src, "-o",
                     str(objs / (Path(src).stem + ".kern.o"))])
    for src in [*map(str, host), str(HERE / "ref_shim.cpp")]:
        jobs.append(["g++", "-std=c++20", "-O3", "-pthread", "-fPIC", *inc, "-c", src, "-o",
                     str(objs / (Path(src).stem + ".host.o"))])
    procs = [subprocess.Popen(c) for c in jobs]
    if any(p.wait() != 0 for p in procs):
        raise RuntimeError("reference build failed")
    cmd = ["g++", "-shared", "-pthread", *[c[-1] for c in jobs], "-o", str(so)]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return so


# The reference's own test programs for this path (tests/CMakeLists.txt:20-26), linked
# against libwake_b200.so instead of the ISPC kernel library.
REFERENCE_TESTS = [
    "unit/test_d2q9_moments.cpp", "unit/test_d2q9_collision.cpp", "unit/test_d3q19_moments.cpp",
    "unit/test_d3q19_collision.cpp", "unit/test_forces_momentum_exchange.cpp",
    "validation/test_poiseuille_convergence.cpp", "validation/test_taylor_green_decay.cpp",
]


def build_reference_tests(lib_dir: Path, verbose: bool = False) -> list[Path]:
    """Compile the reference's hot-path tests from their sources against libwake_b200.so.

    The host sources (LatticeGrid2D/3D, memory, Strouhal) are the reference's, compiled
    unchanged; only the kernel library differs. Asserts stay enabled (no -DNDEBUG).
    Outputs go to oracle/_ref/reftests and find the GPU library via an $ORIGIN rpath.
    """
    ref = reference_dir()
    out_dir = OUT / "reftests"
    out_dir.mkdir(parents=True, exist_ok=True)
    host = [ref / "src" / "grid" / "lattice_grid_2d.cpp", ref / "src" / "grid" / "lattice_grid_3d.cpp",
            ref / "src" / "core" / "memory.cpp", ref / "src" / "forces" / "strouhal_analyzer.cpp",
            ref / "src" / "forces" / "aerodynamic_telemetry.cpp"]
    rel = os.path.relpath(lib_dir, out_dir)
    built = []
    for t in REFERENCE_TESTS:
        exe = out_dir / Path(t).stem
        cmd = ["g++", "-std=c++20", "-O2", f"-I{ref / 'include'}", str(ref / "tests" / t), *map(str, host),
               f"-L{lib_dir}", "-lwake_b200", f"-Wl,-rpath,$ORIGIN/{rel}", "-o", str(exe)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        built.append(exe)
    return built


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
    if "--tests" in sys.argv:
        print(build_reference_tests(HERE.parent / "wake_b200", verbose="-v" in sys.argv))
