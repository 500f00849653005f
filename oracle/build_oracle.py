"""Build recipe for the CPU oracle (test infrastructure only).

Compiles oracle/oracle_capi.cpp with -O2 -ffp-contract=off (no fused multiply-add, matching rustc) into
oracle/liboracle.so (single-threaded checker, the reference's serial loop order) and oracle/liboracle_omp.so
(OpenMP, used only as the timed CPU baseline).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "oracle_capi.cpp")
HDR = os.path.join(HERE, "xpbd_oracle.hpp")
OUT = os.path.join(HERE, "liboracle.so")
OUT_OMP = os.path.join(HERE, "liboracle_omp.so")


def _build_one(out: str, extra: list[str], force: bool) -> str:
    if not force and os.path.exists(out):
        if os.path.getmtime(out) >= max(os.path.getmtime(SRC), os.path.getmtime(HDR)):
            return out
    cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared"] + extra + [
        "-o", out + ".tmp", SRC]
    subprocess.check_call(cmd)
    os.replace(out + ".tmp", out)
    return out


def build(force: bool = False) -> str:
    """Serial checker build (liboracle.so) and the OpenMP build used for the timed CPU baseline
    (liboracle_omp.so: the data-parallel loops of the reference — per constraint, per particle, per color batch —
    run on all host cores; results are identical to the serial build)."""
    _build_one(OUT_OMP, ["-fopenmp"], force)
    return _build_one(OUT, [], force)


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
