"""GPU: fem_plan_assemble_host, the host-buffer assembly with the state upload and
the residual download overlapped with band-split colour launches.  Its schedule
keeps every block's colour order, so residual and matrix must equal
fem_plan_assemble's bit for bit -- on strips of a structured mesh (overlap), on a
mesh whose rows wrap bands unevenly, on scrambled numbering (bands overlap, serial
schedule), for order-1 row assembly, MIXED precision and NONLINEAR strain, and for
any band count."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scramble(fem, m, seed):
    rng = np.random.default_rng(seed)
    perm = rng.permutation(m.num_nodes)
    inv = np.argsort(perm)
    conn = perm[m.conn.reshape(-1, m.nodes_per_element)][rng.permutation(m.num_elements)]
    return fem.Mesh(m.order, np.ascontiguousarray(m.coords[inv]), m.conn_ptr.copy(),
                    np.ascontiguousarray(conn.reshape(-1)).astype(np.int32), np.ascontiguousarray(m.states[inv]),
                    m.E, m.nu, m.t, m.name + "_scrambled", m.seed)


CASES = [
    ("sq40x24_p3", lambda f: f.square_mesh(40, 24, 3, 10.0, 10.0, 0.2, seed=61), "fp64", "linear", 8),
    ("sq40x24_p3_mixed", lambda f: f.square_mesh(40, 24, 3, 10.0, 10.0, 0.2, seed=61), "mixed", "linear", 5),
    ("sq33x17_p2_nl", lambda f: f.square_mesh(33, 17, 2, 1.0, 1.0, 0.1, seed=62), "fp64", "nonlinear", 7),
    ("sq29x31_p4", lambda f: f.square_mesh(29, 31, 4, 1.0, 1.0, 0.1, seed=63), "fp64", "linear", 16),
    ("sq64_p1_rows", lambda f: f.square_mesh(64, 64, 1, 1.0, 1.0, 0.1, seed=64), "fp64", "linear", 8),
    ("scrambled_p3", lambda f: _scramble(f, f.square_mesh(12, 9, 3, 1.0, 1.0, 0.15, seed=65), 65), "fp64", "linear", 6),
    ("annulus_p2", lambda f: f.annulus_mesh(6, 40, 2, seed=66), "mixed", "linear", 1),
]


@pytest.mark.parametrize("layout", ["pairs", "colours"])
@pytest.mark.parametrize("name,make,precision,strain,bands", CASES, ids=[c[0] for c in CASES])
def test_host_assembly_equals_device_assembly(fem, cuda, name, make, precision, strain, bands, layout):
    import torch
    m = make(fem)
    plan = fem.Plan(m.order, m.num_nodes, m.conn_ptr, m.conn)
    if m.order > 1:
        plan.set_layout(layout)  # the band-split launches run the plan's layout
    elif layout == "pairs":
        pytest.skip("order 1: no pair layout")
    d = fem.DeviceMesh(m, cuda)
    res0 = torch.empty(m.num_nodes * 2, dtype=torch.float64, device=cuda)
    mat0 = torch.empty(plan.nnzb * 4, dtype=torch.float64, device=cuda)
    plan.assemble(d.states, d.coords, m.E, m.nu, m.t, res0, mat0, precision=precision, strain=strain)
    h_states = torch.from_numpy(np.ascontiguousarray(m.states).reshape(-1)).pin_memory()
    h_res = torch.full((m.num_nodes * 2,), float("nan"), dtype=torch.float64).pin_memory()
    states = torch.zeros_like(d.states)  # filled by the call
    res = torch.full_like(res0, float("nan"))
    mat = torch.full_like(mat0, float("nan"))
    for _ in range(2):
        secs = plan.assemble_host(h_states, states, d.coords, m.E, m.nu, m.t, h_res, res, mat, precision=precision,
                                  strain=strain, bands=bands, timed=True)
        assert secs > 0
    torch.cuda.synchronize()
    assert torch.equal(states, d.states)
    assert torch.equal(h_res, res0.cpu())
    assert torch.equal(mat, mat0)
    plan.close()


def test_host_assembly_argument_errors(fem, cuda):
    import torch
    m = fem.square_mesh(4, 4, 2, seed=67)
    plan = fem.Plan(2, m.num_nodes, m.conn_ptr, m.conn)
    d = fem.DeviceMesh(m, cuda)
    h = torch.zeros(m.num_nodes * 2, dtype=torch.float64)
    res = torch.zeros(m.num_nodes * 2, dtype=torch.float64, device=cuda)
    with pytest.raises(fem.FemError):
        plan.assemble_host(h, d.states, d.coords, m.E, m.nu, m.t, h, res, None, bands=0)
    with pytest.raises(ValueError):
        plan.assemble_host(d.states, d.states, d.coords, m.E, m.nu, m.t, h, res, None)
    plan.close()
