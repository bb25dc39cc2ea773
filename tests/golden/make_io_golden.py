"""Golden files of the text-I/O tests, written by the reference's own I/O
routines (oracle/ref_io_harness.cpp, built by `make -C oracle ref_io`):

    python tests/golden/make_io_golden.py

Writes tests/golden/io/: the harness's input arrays (in_*.bin, raw float64),
the reference's Print* dumps, WriteRandomMaterial output and what
ReadRandomMaterial read back, a generated Euler-angle texture file and the
orientations ReadRicardoData built from it.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref_io"], check=True)
    out = os.path.join(HERE, "io")
    os.makedirs(out, exist_ok=True)
    subprocess.run([os.path.join(ROOT, "oracle", "_ref", "vpfft_ref_io"), out], check=True,
                   stdout=subprocess.DEVNULL)
    for f in sorted(os.listdir(out)):
        print(f, os.path.getsize(os.path.join(out, f)))


if __name__ == "__main__":
    sys.exit(main())
