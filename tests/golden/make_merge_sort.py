"""Generates tests/golden/merge_sort_cases.npz from merge_sort_cases.cpp
(compiled with g++; libstdc++'s std::mt19937, uniform_int_distribution,
std::merge and std::sort give the inputs and the expected outputs of the
reference's merge and sort tests).

Run:  python tests/golden/make_merge_sort.py
"""
import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "gen")
        subprocess.run(["g++", "-O2", "-std=c++17", "-o", exe, os.path.join(HERE, "merge_sort_cases.cpp")],
                       check=True)
        raw = subprocess.run([exe], check=True, capture_output=True).stdout
    arrays, pos = {}, 0
    while pos < len(raw):
        nl = raw.index(b"\n", pos)
        name = raw[pos:nl].decode()
        (n,) = struct.unpack_from("<q", raw, nl + 1)
        start = nl + 9
        arrays[name] = np.frombuffer(raw, dtype=np.int32, count=n, offset=start).copy()
        pos = start + 4 * n
    np.savez_compressed(os.path.join(HERE, "merge_sort_cases.npz"), **arrays)
    print(f"{len(arrays)} arrays")


if __name__ == "__main__":
    main()
