"""Generates tests/golden/reference_layouts.json: size and member offsets of the
reference's plain data structs (include/core/common.cuh:39-228), measured by
compiling a small host program against the reference's own header with nvcc.
tests/test_cpu_layouts.py compares include/pbs_layouts.h with it.

Usage: python tests/golden/make_layouts.py [--reference <checkout>] [--out <json>]
(the checkout defaults to $REFERENCE_DIR, else <repo>/../reference).
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]

# struct -> members, in the reference's names.
MEMBERS = {
    "vec3f": ["x", "y", "z"],
    "vec3i": ["x", "y", "z"],
    "vec2f": ["x", "y"],
    "Grid": ["corner", "resolution", "upperCorner", "dims"],
    "Source": ["sourcePos", "isoPos", "vsDirX", "vSAD"],
    "Beam": ["source", "bmdir", "bmxdir", "ene", "transCutoff", "longitudalCutoff", "eneIdx"],
    "SubspotInfo": ["deltaX", "deltaY", "weight", "sigmaX", "sigmaY", "eneIdx", "position", "direction",
                    "effectiveSigma", "isValid"],
    "CPBGrid": ["corner", "resolution", "dims", "nLayers"],
}


def program(header_include: str, names: dict | None = None, prelude: str = "") -> str:
    """C/C++ source printing {"struct": {"size": n, "offsets": {...}}} as JSON;
    `names` maps (struct, member) of the reference to the names used by the header."""
    names = names or {}
    lines = [prelude, header_include, "#include <stdio.h>", "#include <stddef.h>", "int main(void) {",
             '  printf("{");']
    for si, (st, mem) in enumerate(MEMBERS.items()):
        tname = names.get(st, st)
        sep = "," if si else ""
        lines.append(f'  printf("{sep}\\"{st}\\": {{\\"size\\": %zu, \\"offsets\\": {{", sizeof({tname}));')
        for mi, m in enumerate(mem):
            mname = names.get((st, m), m)
            msep = "," if mi else ""
            lines.append(f'  printf("{msep}\\"{m}\\": %zu", offsetof({tname}, {mname}));')
        lines.append('  printf("}}");')
    lines += ['  printf("}\\n");', "  return 0;", "}"]
    return "\n".join(lines)


def measure(source: str, compiler: list, suffix: str) -> dict:
    with tempfile.TemporaryDirectory() as d:
        src = Path(d) / f"layouts{suffix}"
        exe = Path(d) / "layouts"
        src.write_text(source)
        subprocess.run([*compiler, str(src), "-o", str(exe)], check=True, capture_output=True)
        out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return json.loads(out)


def reference_layouts(checkout: Path) -> dict:
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    inc = [f"-I{checkout / 'include'}", f"-I{checkout / 'include' / 'core'}", f"-I{checkout / 'include' / 'utils'}"]
    src = program('#include "common.cuh"')
    return measure(src, [nvcc, "-std=c++17", "-w", *inc], ".cu")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("REFERENCE_DIR", str(ROOT.parent / "reference")))
    ap.add_argument("--out", default=str(Path(__file__).resolve().parent / "reference_layouts.json"))
    a = ap.parse_args(argv)
    lay = reference_layouts(Path(a.reference))
    Path(a.out).write_text(json.dumps({"source": "include/core/common.cuh:39-228 of Nelgcis/subsecondPBS, "
                                       "measured by tests/golden/make_layouts.py", "layouts": lay}, indent=1) + "\n")
    print(json.dumps(lay))
    return 0


if __name__ == "__main__":
    sys.exit(main())
