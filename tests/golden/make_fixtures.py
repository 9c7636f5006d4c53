"""Regenerate the reference-pinned fixtures in this folder.

Runs oracle/_ref/ref_driver (the reference's own build_tree.cpp compiled from
its source tree by oracle/Makefile, plus its header-only test_funcs.hpp and
kernel.hpp) and stores its points, right-hand side, tree, Near/Far lists,
kernel values (Laplace, Yukawa, Helmholtz) and mesh_sphere points as .npz files.  Needs the reference source tree, so it runs in
the development container only; the fixtures it writes are committed.

    make -C oracle && python tests/golden/make_fixtures.py
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")

CASES = [
    # name, N, leaf, theta, seed
    ("ref_n2048_leaf256_theta2_seed999", 2048, 256, 2.0, 999),
    ("ref_n5000_leaf128_theta1.5_seed7", 5000, 128, 1.5, 7),
    ("ref_n300_leaf512_theta2_seed3", 300, 512, 2.0, 3),
]


def read_dump(path: str) -> dict:
    raw = open(path, "rb").read()
    off = 0

    def ints(n):
        nonlocal off
        v = np.frombuffer(raw, dtype=np.int64, count=n, offset=off).copy()
        off += 8 * n
        return v

    def dbls(n):
        nonlocal off
        v = np.frombuffer(raw, dtype=np.float64, count=n, offset=off).copy()
        off += 8 * n
        return v

    N, levels, ncells = (int(v) for v in ints(3))
    out = {"N": N, "levels": levels}
    out["bodies"] = dbls(3 * N).reshape(N, 3)
    out["xbody"] = dbls(N)
    child = np.zeros((ncells, 2), np.int64)
    body = np.zeros((ncells, 2), np.int64)
    R = np.zeros((ncells, 3))
    C = np.zeros((ncells, 3))
    for c in range(ncells):
        a = ints(4)
        child[c], body[c] = a[:2], a[2:]
        R[c] = dbls(3)
        C[c] = dbls(3)
    out.update(child=child, body=body, R=R, C=C)
    for name in ("near", "far", "far0"):
        nr = int(ints(1)[0])
        row = ints(nr)
        nz = int(ints(1)[0])
        col = ints(nz)
        out[name + "_row"] = row
        out[name + "_col"] = col
    npairs = int(ints(1)[0])
    ij = np.zeros((npairs, 2), np.int64)
    vals = np.zeros((npairs, 2))
    for k in range(npairs):
        ij[k] = ints(2)
        vals[k] = dbls(2)
    out["probe_ij"] = ij
    out["probe_laplace"] = vals[:, 0]
    out["probe_yukawa"] = vals[:, 1]
    nh = int(ints(1)[0])
    hv = dbls(2 * nh).reshape(nh, 2)
    out["probe_helmholtz"] = hv[:, 0] + 1j * hv[:, 1]
    ns = int(ints(1)[0])
    out["mesh_sphere"] = dbls(3 * ns).reshape(ns, 3)
    return out


def main() -> int:
    if not os.path.exists(DRIVER):
        print("build the driver first: make -C oracle", file=sys.stderr)
        return 1
    for name, N, leaf, theta, seed in CASES:
        with tempfile.TemporaryDirectory() as td:
            dump = os.path.join(td, "d.bin")
            subprocess.run([DRIVER, str(N), str(leaf), str(theta), str(seed), dump], check=True)
            d = read_dump(dump)
        d.update(leaf=leaf, theta=theta, seed=seed)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **d)
        print("wrote", name)
    return 0


if __name__ == "__main__":
    sys.exit(main())
