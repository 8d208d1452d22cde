"""TEST INFRASTRUCTURE: writes the two generated headers the reference's sources expect when they are compiled
unmodified into oracle/_ref/ (see oracle/Makefile):

* ``cambi_lut.h``: ``__constant__ float reciprocal_lut[4226]`` with entry i = 1/i as a float (entry 0 = 0), the table
  the reference's build copies from libvmaf (reference scripts/container-build.sh:30-32); the values are printed with
  9 significant digits, which round-trip a float exactly;
* ``kernels_fatbin.h``: the compiled reference kernels as ``unsigned char kernels_fatbin[]`` (what the reference's
  build makes with ``xxd -i``, scripts/container-build.sh:36-37), included by its src/gpu.cpp.

Usage: gen_ref_headers.py lut OUT.h | gen_ref_headers.py fatbin IN.fatbin OUT.h
"""

import sys

import numpy as np


def lut(out: str) -> None:
    n = 4226
    def literal(x: np.float32) -> str:
        s = f"{x:.9g}"
        return (s if ("." in s or "e" in s) else s + ".0") + "f"

    vals = ["0.0f"] + [literal(np.float32(1.0) / np.float32(i)) for i in range(1, n)]
    body = ",\n".join(", ".join(vals[i:i + 8]) for i in range(0, n, 8))
    with open(out, "w") as f:
        f.write(f"// generated by oracle/gen_ref_headers.py: reciprocal_lut[i] = 1/i\n__constant__ float reciprocal_lut[{n}] = {{\n{body}\n}};\n")


def fatbin(src: str, out: str) -> None:
    data = open(src, "rb").read()
    rows = [", ".join(f"0x{b:02x}" for b in data[i:i + 16]) for i in range(0, len(data), 16)]
    with open(out, "w") as f:
        f.write("// generated by oracle/gen_ref_headers.py from the reference kernels built for sm_100a\n")
        f.write("unsigned char kernels_fatbin[] = {\n" + ",\n".join(rows) + "\n};\n")
        f.write(f"unsigned int kernels_fatbin_len = {len(data)};\n")


if __name__ == "__main__":
    if sys.argv[1] == "lut":
        lut(sys.argv[2])
    elif sys.argv[1] == "fatbin":
        fatbin(sys.argv[2], sys.argv[3])
    else:
        raise SystemExit(__doc__)
