"""Build the oracle's C restatement (oracle/_ref is not used: the reference is
Rust and cannot be built here; this is the C port)."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "libsocs_cpu.so")


def build() -> str:
    src = os.path.join(HERE, "socs_cpu.c")
    if os.path.exists(SO) and os.path.getmtime(SO) >= os.path.getmtime(src):
        return SO
    subprocess.run(["gcc", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fPIC", "-shared", "-o", SO, src,
                    "-lpthread", "-lm"], check=True)
    return SO


if __name__ == "__main__":
    print(build())
