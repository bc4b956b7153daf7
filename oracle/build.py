"""Build recipe for the C part of the oracle (test infrastructure only).

    python -m oracle.build      ->  oracle/_build/liboracle.so
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(force: bool = False) -> str:
    out_dir = os.path.join(HERE, "_build")
    os.makedirs(out_dir, exist_ok=True)
    out = os.path.join(out_dir, "liboracle.so")
    src = os.path.join(HERE, "xatu_oracle.c")
    if not force and os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(src):
        return out
    cmd = ["gcc", "-O2", "-Wall", "-Werror=implicit-function-declaration", "-fopenmp", "-fPIC", "-shared", "-std=c11", "-o", out, src, "-lm"]
    subprocess.run(cmd, check=True)
    return out


if __name__ == "__main__":
    print(build(force=True))
