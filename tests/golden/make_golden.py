"""Regenerate the fixtures in this folder from the reference checkout (run where the reference is available).

    python tests/golden/make_golden.py /path/to/bevy_xpbd

cloth.obj — the reference's own asset `assets/cloth.obj` (a 21 x 31 vertex Blender grid, MIT licence of
mate-h/bevy_xpbd), copied byte for byte. It is the one input fixture the reference ships for this path; the tests parse
it through `parse_welded_obj` (src/mesh_prep.rs:223-357) in the product and in the oracle and step it on the GPU.
The reference cannot be built here (no Rust toolchain), so no reference outputs are stored: the expected structure of
the parsed mesh is derived from the reference source in tests/test_golden_cpu.py.
"""
import hashlib
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root: str) -> None:
    src = os.path.join(ref_root, "assets", "cloth.obj")
    dst = os.path.join(HERE, "cloth.obj")
    shutil.copyfile(src, dst)
    with open(dst, "rb") as f:
        print("cloth.obj sha256", hashlib.sha256(f.read()).hexdigest())


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
