"""Build recipe: compile the reference's own CUDA-C kernels as a CPU shared library.

TEST INFRASTRUCTURE ONLY (oracle).  The product never imports, links or runs this.

The reference keeps all of its device code in one CUDA-C string passed to
``pycuda.compiler.SourceModule`` (mainPropElastic3D_MT.py:42-514).  This recipe
reads that string from the read-only reference tree at build time, writes it (plus
generated ``extern "C"`` launch wrappers, one per ``__global__`` function) into
``oracle/_ref/`` -- which git ignores, so no reference source enters the repository --
and compiles it with ``g++ -fopenmp`` through :file:`oracle/ref_shim.h`, which maps the
CUDA built-ins onto host loops.

Outputs (all under ``oracle/_ref/``):

* ``librefkern.so``      -- ``ref_<kernel>(grid[3], block[3], parallel, <kernel args>)``
* ``signatures.json``    -- kernel name -> list of (c_type, name), for ctypes callers
* ``kernels.sha256``     -- hash of the kernel string, so callers can check they drive
                            exactly the compiled source.

Run: ``python oracle/build_ref.py`` (needs the reference tree; a no-op when the
library is up to date).
"""
from __future__ import annotations

import hashlib
import json
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
REF_FILE = os.environ.get(
    "EFM_REFERENCE_MAIN",
    "/root/reference/Elastic3DGPU_MT_VP_VS_RHO_MPI/mainPropElastic3D_MT.py",
)

_KERNEL_RE = re.compile(r"__global__\s+void\s+(\w+)\s*\(([^)]*)\)", re.S)


def extract_kernel_source(path: str = REF_FILE) -> str:
    """Return the CUDA-C string handed to SourceModule (mainPropElastic3D_MT.py:42-514)."""
    with open(path, "r", encoding="utf-8") as f:
        text = f.read()
    m = re.search(r'SourceModule\(\s*"""(.*?)"""\s*\)', text, re.S)
    if m is None:
        raise RuntimeError(f"no SourceModule(\"\"\"...\"\"\") string found in {path}")
    return m.group(1)


def parse_signatures(src: str) -> dict[str, list[tuple[str, str]]]:
    """Map each __global__ function to its (type, name) parameter list."""
    sigs: dict[str, list[tuple[str, str]]] = {}
    for name, params in _KERNEL_RE.findall(src):
        plist = []
        for p in params.split(","):
            p = " ".join(p.split())
            if not p:
                continue
            m = re.match(r"(.*?)([A-Za-z_]\w*)$", p)
            ctype = m.group(1).replace(" ", "")
            plist.append((ctype, m.group(2)))
        sigs[name] = plist
    return sigs


def _wrappers(sigs: dict[str, list[tuple[str, str]]]) -> str:
    lines = []
    for name, params in sigs.items():
        decl = ", ".join(f"{t.replace('*', ' *')} {n}" for t, n in params)
        call = ", ".join(n for _, n in params)
        lines.append(
            f'extern "C" void ref_{name}(const unsigned *grid, const unsigned *block, int parallel'
            + (f", {decl}" if decl else "")
            + ") {\n"
            f"    efm_ref_launch(grid, block, parallel != 0, [&]() {{ {name}({call}); }});\n"
            "}\n"
        )
    return "\n".join(lines)


def build(force: bool = False, quiet: bool = True) -> str:
    """Compile ``oracle/_ref/librefkern.so``; return its path."""
    src = extract_kernel_source()
    digest = hashlib.sha256(src.encode()).hexdigest()
    so = os.path.join(OUT, "librefkern.so")
    stamp = os.path.join(OUT, "kernels.sha256")
    if (not force and os.path.exists(so) and os.path.exists(stamp)
            and open(stamp).read().strip() == digest):
        return so
    os.makedirs(OUT, exist_ok=True)
    sigs = parse_signatures(src)
    unit = os.path.join(OUT, "ref_kernels_host.cpp")
    with open(unit, "w") as f:
        f.write('#include "ref_shim.h"\n')
        f.write(src)
        f.write("\n\n")
        f.write(_wrappers(sigs))
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
           "-w", f"-I{HERE}", unit, "-o", so]
    subprocess.run(cmd, check=True, capture_output=quiet)
    with open(os.path.join(OUT, "signatures.json"), "w") as f:
        json.dump(sigs, f, indent=1)
    with open(stamp, "w") as f:
        f.write(digest + "\n")
    return so


if __name__ == "__main__":
    path = build(force="--force" in sys.argv, quiet=False)
    print(path)
