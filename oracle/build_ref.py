"""Recipe: the reference's C example caller, compiled unchanged.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Compiles LibNEGF.jl's ``src/c_interface/libnegf_c_example.c`` against its own
header ``libnegf_c_interface.h`` where they lie in the reference checkout,
with ``oracle/c_example_wrap.c`` as a link-time probe around
``run_bndiag_wrapper`` (``-Wl,--wrap``), and links it to this repository's
``libnegf_b200.so``.  Output: ``oracle/_ref/libnegf_c_example`` (git-ignored;
it travels with the repository to the GPU machine).  Nothing is copied from
the reference into the repository.

    python oracle/build_ref.py [reference root]
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT_DIR = os.path.join(HERE, "_ref")
LIB_DIR = os.path.join(ROOT, "libnegf.jl_b200", "libnegf_b200")


def build_c_example(ref_root="/root/reference"):
    src_dir = os.path.join(ref_root, "src", "c_interface")
    src = os.path.join(src_dir, "libnegf_c_example.c")
    if not os.path.exists(src):
        return None
    os.makedirs(OUT_DIR, exist_ok=True)
    out = os.path.join(OUT_DIR, "libnegf_c_example")
    rpath = "$ORIGIN/" + os.path.relpath(LIB_DIR, OUT_DIR)
    cmd = ["gcc", "-O2", "-std=c11", "-I" + src_dir, src, os.path.join(HERE, "c_example_wrap.c"),
           "-Wl,--wrap=run_bndiag_wrapper", "-L" + LIB_DIR, "-l:libnegf_b200.so", "-Wl,-rpath," + rpath, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("building the reference C example failed:\n" + r.stderr)
    return out


if __name__ == "__main__":
    print(build_c_example(*sys.argv[1:]))
