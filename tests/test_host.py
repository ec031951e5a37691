"""CPU tests of the library's host side: the C ABI loads and exports every
declared symbol, and the integer topology work (BSR pattern, element->block
map, colouring) is bit-exact against the oracle's independent restatement."""
import pathlib
import re

import numpy as np
import pytest

HEADER = pathlib.Path(__file__).resolve().parent.parent / "include" / "fem_b200.h"


def _declared():
    txt = HEADER.read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(fem_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(fem):
    names = _declared()
    assert len(names) >= 15
    missing = [n for n in names if getattr(fem.lib, n, None) is None]
    assert not missing, missing
    assert fem.lib.fem_version() >= 100


def test_probe_library_exports_its_symbols(fem):
    """The arithmetic-peak probes live in libfemprobe.so (include/fem_probe.h),
    outside the assembly library's interface."""
    import ctypes as C
    txt = re.sub(r"/\*.*?\*/", "", (HEADER.parent / "fem_probe.h").read_text(), flags=re.S)
    names = sorted(set(re.findall(r"\b(fem_[a-z0-9_]+)\s*\(", txt)))
    assert names == ["fem_probe_peak"]
    probe = C.CDLL(str(pathlib.Path(fem.lib._name).parent / "libfemprobe.so"))
    assert all(getattr(probe, n, None) is not None for n in names)
    assert getattr(fem.lib, "fem_probe_peak", None) is None


def test_python_mirror_binds_every_declared_symbol(fem):
    """The ctypes table of the host mirror covers the whole C ABI (argument types
    set for every entry point the header declares)."""
    from importlib import import_module
    lib_mod = import_module(fem.__name__ + "._lib")
    missing = [n for n in _declared() if n not in lib_mod.SIGNATURES]
    assert not missing, missing


def test_status_strings(fem):
    for s in range(0, 9):
        assert fem.lib.fem_status_string(s)


MESHES = [
    ("sq_p1", lambda f: f.square_mesh(7, 5, 1, 1.0, 1.0, 0.1, seed=1)),
    ("sq_p2", lambda f: f.square_mesh(4, 6, 2, 1.0, 2.0, 0.2, seed=2)),
    ("sq_p3", lambda f: f.square_mesh(3, 3, 3, seed=3)),
    ("sq_p4", lambda f: f.square_mesh(2, 3, 4, seed=4)),
    ("ann_p2", lambda f: f.annulus_mesh(2, 9, 2, seed=5)),
    ("one_el", lambda f: f.square_mesh(1, 1, 3, seed=6)),
    ("strip", lambda f: f.square_mesh(9, 1, 1, seed=7)),
]


@pytest.mark.parametrize("name,make", MESHES)
def test_pattern_map_colour_bit_exact(fem, orc, name, make):
    m = make(fem)
    n = m.nodes_per_element
    rowp, cols = fem.build_bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
    r2, c2 = orc.bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
    assert np.array_equal(rowp, r2) and np.array_equal(cols, c2)
    mp = fem.build_element_bsr_map(m.conn_ptr, m.conn, n, rowp, cols)
    assert np.array_equal(mp, orc.element_bsr_map(m.conn_ptr, m.conn, n, r2, c2))
    colour, nc = fem.colour_elements(m.num_nodes, m.conn_ptr, m.conn)
    assert orc.check_colouring(m.num_nodes, m.conn_ptr, m.conn, colour, nc) == 0
    assert colour.min() == 0 and colour.max() == nc - 1


def test_structured_pattern_counts(fem):
    """nnzb of an nx x ny order-p structured mesh is (nx(p^2+2p)+1)(ny(p^2+2p)+1)."""
    for p in range(1, 5):
        m = fem.square_mesh(5, 3, p)
        rowp, cols = fem.build_bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
        assert cols.size == (5 * (p * p + 2 * p) + 1) * (3 * (p * p + 2 * p) + 1)
    m = fem.square64_p1()
    rowp, cols = fem.build_bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
    assert cols.size == 193 ** 2


def test_structured_colouring_is_four_colours(fem):
    m = fem.square_mesh(10, 7, 2)
    _, nc = fem.colour_elements(m.num_nodes, m.conn_ptr, m.conn)
    assert nc == 4


def test_colouring_is_deterministic(fem):
    m = fem.annulus_mesh(4, 16, 1, seed=2)
    a, na = fem.colour_elements(m.num_nodes, m.conn_ptr, m.conn)
    b, nb = fem.colour_elements(m.num_nodes, m.conn_ptr, m.conn)
    assert na == nb and np.array_equal(a, b)


def test_host_errors(fem):
    m = fem.square_mesh(2, 2, 1)
    bad = m.conn.copy()
    bad[3] = m.num_nodes  # out of range
    with pytest.raises(fem.FemError) as ei:
        fem.build_bsr_pattern(m.num_nodes, m.conn_ptr, bad)
    assert ei.value.status == fem.FEM_ERR_INVALID_ARGUMENT
    rowp, cols = fem.build_bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
    cols2 = cols.copy()
    cols2[rowp[4]] = -1 if cols2[rowp[4]] != 0 else 10 ** 6  # corrupt one row
    with pytest.raises(fem.FemError) as ei:
        fem.build_element_bsr_map(m.conn_ptr, m.conn, 4, rowp, np.sort(cols2))
    assert ei.value.status == fem.FEM_ERR_NOT_FOUND


def test_empty_mesh(fem):
    rowp, cols = fem.build_bsr_pattern(3, np.zeros(1, np.int32), np.zeros(0, np.int32))
    assert rowp.tolist() == [0, 0, 0, 0] and cols.size == 0
    colour, nc = fem.colour_elements(3, np.zeros(1, np.int32), np.zeros(0, np.int32))
    assert nc == 0 and colour.size == 0


def test_device_entry_points_refuse_cpu_tensors(fem):
    torch = pytest.importorskip("torch")
    m = fem.square_mesh(2, 2, 1)
    t = torch.zeros(10, dtype=torch.float64)
    with pytest.raises(ValueError):
        fem.run_residual_kernel(1, torch.from_numpy(m.conn_ptr), torch.from_numpy(m.conn), 4, t, t, 1.0, 0.3, 1.0, t,
                                stream=0)
