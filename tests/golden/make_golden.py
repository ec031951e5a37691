"""Regenerates the committed golden vectors from the reference's own code.

* ref_tables.txt: the Gauss and shape-derivative tables computed by the
  reference's element/GaussQuadrature.h and element/LagrangeShapeFuncs.h
  (oracle/_ref/ref_tables, exact hexadecimal floats).
* ref_assembly.npz: inputs and outputs of the reference's CPU assembly
  (runResidualKernel / runJacobianKernel, element/FEKernels.h:317-508 and
  :1030-1225, compiled from the header as oracle/_ref/libfemref.so against the
  A2D interface restated in oracle/a2d_shim/): small meshes of orders 1 to 4
  (squares and an annulus, LINEAR residual and Jacobian, NONLINEAR residual),
  and for the 64x64 order-1 mesh the residual, the matrix applied to a seeded
  vector and the matrix's Frobenius norm.

Both programs are built by oracle/Makefile (target `ref`, which reads the
reference checkout).  Usage: python tests/golden/make_golden.py [REF=<checkout>]
"""
import pathlib
import subprocess
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

# small meshes: (name, builder arguments); every array they produce is stored
SMALL = [
    ("sq_p1", dict(nx=5, ny=4, p=1, lx=1.0, ly=1.0, perturb=0.1, seed=0x601)),
    ("sq_p2", dict(nx=4, ny=3, p=2, lx=2.0, ly=1.0, perturb=0.15, seed=0x602)),
    ("sq_p3", dict(nx=3, ny=3, p=3, lx=10.0, ly=10.0, perturb=0.2, seed=0x603)),
    ("sq_p4", dict(nx=3, ny=2, p=4, lx=1.0, ly=1.5, perturb=0.15, seed=0x604)),
]
ANNULUS = ("an_p2", dict(nr=2, nth=8, p=2, seed=0x605))
CONFIG1_VECTOR_SEED = 0x60A


def main():
    make = ["make", "-s", "-C", str(ROOT / "oracle"), "ref"] + [a for a in sys.argv[1:] if a.startswith("REF=")]
    subprocess.run(make, check=True)
    out = subprocess.run([str(ROOT / "oracle" / "_ref" / "ref_tables")], check=True, capture_output=True, text=True)
    (HERE / "ref_tables.txt").write_text(out.stdout)

    import fem_pkg
    import oracle as orc
    mesh = fem_pkg.load_module("mesh")
    arrays = {}

    def store(name, m, full=True):
        rowp, cols = orc.bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
        mp = orc.element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols)
        R, A = orc.ref_assemble(m, mp, cols.size)
        Rn, _ = orc.ref_assemble(m, jacobian=False, strain="nonlinear")
        arrays[f"{name}/material"] = np.array([m.order, m.num_nodes, m.E, m.nu, m.t])
        arrays[f"{name}/residual"] = R
        arrays[f"{name}/residual_nonlinear"] = Rn
        if full:
            for k, v in (("coords", m.coords), ("states", m.states), ("conn_ptr", m.conn_ptr), ("conn", m.conn),
                         ("rowp", rowp), ("cols", cols), ("matrix", A)):
                arrays[f"{name}/{k}"] = np.ascontiguousarray(v)
        else:
            v = np.random.default_rng(CONFIG1_VECTOR_SEED).uniform(-1.0, 1.0, m.num_nodes * 2)
            arrays[f"{name}/matvec"] = orc.bsr_spmv(rowp, cols, A, v)
            arrays[f"{name}/matrix_fro"] = np.array([np.linalg.norm(A)])

    for name, kw in SMALL:
        store(name, mesh.square_mesh(**kw))
    store(ANNULUS[0], mesh.annulus_mesh(**ANNULUS[1]))
    store("config1", mesh.square64_p1(), full=False)
    np.savez_compressed(HERE / "ref_assembly.npz", **arrays)
    print(f"wrote {HERE / 'ref_tables.txt'} and {HERE / 'ref_assembly.npz'} ({len(arrays)} arrays)")


if __name__ == "__main__":
    main()
