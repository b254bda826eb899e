"""Generates sobol_1024x52.bin, the Sobol generator matrices used by the device
Z-Sobol sampler.

Restates Sources/SobolGenerator/main.swift:11-76 of Gonzales: 1024 dimensions x
52 uint32 columns, dimension 0 the bit-reversal (van der Corput) matrix and
dimensions 1..1023 from the Joe-Kuo direction numbers (Joe & Kuo, "Constructing
Sobol sequences with better two-dimensional projections", SIAM J. Sci. Comput.
30(5), 2008; file new-joe-kuo-6.21201, shipped by Gonzales as
Sources/libgonzales/Resources/new-joe-kuo-6.21201).  The table is stored
little-endian, dimension-major, exactly as the generator's base64 payload.

Usage: python gen_sobol_matrices.py <new-joe-kuo-6.21201> [out.bin]
"""
import struct
import sys
from pathlib import Path

N_DIMS = 1024
MATRIX_SIZE = 52
MASK32 = 0xFFFFFFFF


def parse_direction_numbers(text):
    entries = []
    for line in text.splitlines():
        line = line.strip()
        if not line or line.startswith("d"):
            continue
        parts = line.split()
        if len(parts) < 3:
            continue
        s, a = int(parts[1]), int(parts[2])
        m = [int(x) for x in parts[3:]]
        entries.append((s, a, m))
    return entries


def generate(entries):
    mats = [[0] * MATRIX_SIZE for _ in range(N_DIMS)]
    for i in range(32):
        mats[0][i] = 1 << (31 - i)
    for dim in range(1, N_DIMS):
        if dim - 1 >= len(entries):
            break
        s, a, m = entries[dim - 1]
        v = [0] * (MATRIX_SIZE + 1)
        for i in range(1, s + 1):
            v[i] = (m[i - 1] << (32 - i)) & MASK32
        for i in range(s + 1, MATRIX_SIZE + 1):
            v[i] = v[i - s] ^ (v[i - s] >> s)
            for j in range(1, s):
                if (a >> (s - 1 - j)) & 1 == 1:
                    v[i] ^= v[i - j]
            v[i] &= MASK32
        for i in range(MATRIX_SIZE):
            mats[dim][i] = v[i + 1]
    return mats


def to_bytes(mats):
    return b"".join(struct.pack("<%dI" % MATRIX_SIZE, *row) for row in mats)


def main():
    src = Path(sys.argv[1])
    out = Path(sys.argv[2]) if len(sys.argv) > 2 else Path(__file__).with_name("sobol_1024x52.bin")
    mats = generate(parse_direction_numbers(src.read_text()))
    out.write_bytes(to_bytes(mats))
    print(f"wrote {out} ({N_DIMS} dims x {MATRIX_SIZE})")


if __name__ == "__main__":
    main()
