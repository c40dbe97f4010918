"""Regenerates tests/golden/sort_mt19937_3.npz from sort_golden.cpp (g++ required).

n = 1, 2, 1000 are stored in full; n = 100000 as the input keys (400 KB compressed well below
that: the keys are stored, the expected order as a SHA-256 of the sorted key and value bytes)."""
import hashlib
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "sort_golden")
        subprocess.run(["g++", "-O2", "-std=c++17", os.path.join(HERE, "sort_golden.cpp"), "-o", exe], check=True)
        subprocess.run([exe, tmp], check=True)
        out = {}
        for n in (1, 2, 1000, 100000):
            load = lambda s: np.fromfile(os.path.join(tmp, f"sort_n{n}_{s}.bin"), dtype="<u4")
            keys, sk, sv = load("keys"), load("sorted_keys"), load("sorted_values")
            out[f"n{n}_keys"] = keys
            if n <= 1000:
                out[f"n{n}_sorted_keys"] = sk
                out[f"n{n}_sorted_values"] = sv
            digest = hashlib.sha256(sk.tobytes() + sv.tobytes()).hexdigest()
            out[f"n{n}_sha256"] = np.frombuffer(bytes.fromhex(digest), dtype=np.uint8)
        np.savez_compressed(os.path.join(HERE, "sort_mt19937_3.npz"), **out)


if __name__ == "__main__":
    main()
