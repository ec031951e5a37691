"""Loader of tests/golden/ref_assembly.npz: meshes and outputs of the reference's
own CPU assembly (element/FEKernels.h compiled as oracle/_ref/libfemref.so by
tests/golden/make_golden.py)."""
import pathlib

import numpy as np

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden" / "ref_assembly.npz"
SMALL = ("sq_p1", "sq_p2", "sq_p3", "sq_p4", "an_p2")


def load():
    return np.load(GOLDEN)


def mesh(z, name):
    """The stored mesh `name` as a mesh.Mesh."""
    import fem_pkg
    Mesh = fem_pkg.load_module("mesh").Mesh
    order, _, E, nu, t = z[f"{name}/material"]
    return Mesh(int(order), z[f"{name}/coords"], z[f"{name}/conn_ptr"], z[f"{name}/conn"], z[f"{name}/states"],
                float(E), float(nu), float(t), name)


def rel(a, b):
    """Normwise relative difference max|a - b| / max|b|."""
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))
