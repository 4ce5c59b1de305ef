"""Regenerates the committed golden vectors of tests/golden.

well19937a_*.txt  first draws of the reference's own WELL19937a generator (src/WELL19937a_new.c compiled in
                  place by oracle/Makefile into oracle/_ref/libwell_ref.so), seeded through the restated
                  well_random_seed of pic2d_RandomNumberInterface.f90:39-57 (the seeding words are built here in
                  Python, independently of the oracle). These pin the oracle's restated generator.
Run from the repository root after `make -C oracle`:  python tests/golden/make_golden.py
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, "..", "..", "oracle", "_ref", "libwell_ref.so")


def seed_words(seed):
    w = [seed & 0xFFFFFFFF]
    for j in range(1, 624):
        x = w[-1]
        w.append((1812433253 * ((x ^ (x << 30)) & 0xFFFFFFFF) + j) & 0xFFFFFFFF)
    return w


def reference_stream(seed, n):
    lib = C.CDLL(REF)
    words = (C.c_uint * 624)(*seed_words(seed))
    si, fn = C.c_uint(0), C.c_uint(1)
    lib.set_state(words, C.byref(si), C.byref(fn))
    f = C.CFUNCTYPE(C.c_double)
    return [f(C.c_void_p.in_dll(lib, "WELLRNG19937").value)() for _ in range(n)]


if __name__ == "__main__":
    for seed in (123456789, 0, 2147483647, -5):
        vals = reference_stream(seed, 2000)
        with open(os.path.join(HERE, f"well19937a_{seed}.txt"), "w") as fh:
            fh.write(f"# first 2000 draws of WELL19937a_new.c after well_random_seed({seed})\n")
            fh.writelines(f"{v.hex()}\n" for v in vals)
    print("written")
