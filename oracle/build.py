"""Builds the oracle's C++ helper with g++ (test infrastructure only)."""
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))


def build_oracle():
    out_dir = os.path.join(_HERE, "_build")
    os.makedirs(out_dir, exist_ok=True)
    src = os.path.join(_HERE, "rng.cpp")
    out = os.path.join(out_dir, "liboracle_rng.so")
    if os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(src):
        return out
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-shared", "-fPIC",
                           src, "-o", out])
    return out


if __name__ == "__main__":
    print(build_oracle())
