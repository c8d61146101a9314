"""Writes mc_reference_tables.npz: the reference's marching-cubes case tables
(gaussrecon_src/MarchingCubes.cpp:32-324, edgeMask[256] and triangles[256][16])
read out of the reference's own code compiled by `make -C oracle ref-mc`
(oracle/_ref/libref_mc.so).  They feed the caller-supplied-table mode of
cagr_marching_cubes_table in the tests, which need neither the reference
checkout nor its build at test time.

    make -C oracle ref-mc && python tests/golden/make_mc_tables.py
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
LIB = os.path.join(ROOT, "oracle", "_ref", "libref_mc.so")


def main() -> None:
    if not os.path.exists(LIB):
        sys.exit("build the reference's marching cubes first: make -C oracle ref-mc")
    lib = ctypes.CDLL(LIB)
    edge_mask = np.zeros(256, np.int32)
    triangles = np.zeros(256 * 16, np.int32)
    lib.ref_mc_tables(edge_mask.ctypes.data_as(ctypes.c_void_p),
                      triangles.ctypes.data_as(ctypes.c_void_p))
    np.savez_compressed(os.path.join(HERE, "mc_reference_tables.npz"),
                        edge_mask=edge_mask, triangles=triangles.reshape(256, 16).astype(np.int8))
    print("wrote mc_reference_tables.npz")


if __name__ == "__main__":
    main()
