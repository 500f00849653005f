"""Build recipe for the CPU oracle (test infrastructure only).

Compiles oracle/oracle_capi.cpp into oracle/liboracle.so with -O2 -ffp-contract=off (no fused multiply-add,
matching rustc), and an OpenMP-free single-threaded build so the FP32 oracle follows the reference's serial
loop order exactly.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "oracle_capi.cpp")
HDR = os.path.join(HERE, "xpbd_oracle.hpp")
OUT = os.path.join(HERE, "liboracle.so")


def build(force: bool = False) -> str:
    if not force and os.path.exists(OUT):
        if os.path.getmtime(OUT) >= max(os.path.getmtime(SRC), os.path.getmtime(HDR)):
            return OUT
    cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
           "-o", OUT + ".tmp", SRC]
    subprocess.check_call(cmd)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
