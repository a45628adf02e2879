"""Build the CPU oracle (oracle/_build/liboracle.so).  Test infrastructure."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_build", "liboracle.so")


def build():
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    src = os.path.join(HERE, "sdft_oracle.c")
    if os.path.exists(OUT) and os.path.getmtime(OUT) > max(os.path.getmtime(src),
                                                            os.path.getmtime(os.path.join(HERE, "sdft_oracle.h"))):
        return OUT
    subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-ffp-contract=off", src, "-o", OUT, "-lm"], check=True)
    return OUT


if __name__ == "__main__":
    print(build())
