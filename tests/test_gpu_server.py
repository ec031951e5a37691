"""GPU: the continuous-batching assembly server.  Each request's result is the
same alone and in a mix of concurrent requests (bit for bit, and within the FP64
tolerance of the oracle), admission respects the device-memory budget, and many
client threads can submit concurrently."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _meshes(fem):
    specs = fem.batch_specs(count=10, lo=4, hi=400, seed=77)
    return [s.build() for s in specs]


def _alone(fem, cuda, m, x, precision):
    """Residual and A*x of m assembled by its own plan (single-mesh path)."""
    import torch
    p = fem.Plan(m.order, m.num_nodes, m.conn_ptr, m.conn)
    if m.order > 1:
        p.set_layout("colours")  # the server runs the colour layout
    d = fem.DeviceMesh(m, cuda)
    r = torch.empty(m.num_nodes * 2, dtype=torch.float64, device=cuda)
    a = torch.empty(p.nnzb * 4, dtype=torch.float64, device=cuda)
    p.assemble(d.states, d.coords, m.E, m.nu, m.t, r, a, precision=precision)
    rowp, cols = p.device_pattern()
    y = torch.empty_like(x)
    fem.lib.fem_bsr_spmv(m.num_nodes, rowp, cols, a.data_ptr(), x.data_ptr(), y.data_ptr(),
                         torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    out = (r.cpu(), y.cpu())
    p.close()
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_results_same_alone_and_in_the_mix(fem, orc, cuda, precision):
    import torch
    meshes = _meshes(fem)
    srv = fem.Server(8 << 30, precision=precision, max_batch=64)
    ids = [srv.add_mesh(m) for m in meshes]
    states = [torch.from_numpy(np.ascontiguousarray(m.states)).pin_memory() for m in meshes]
    res_mix = [torch.empty(m.num_nodes * 2, dtype=torch.float64).pin_memory() for m in meshes]
    res_alone = [torch.empty(m.num_nodes * 2, dtype=torch.float64).pin_memory() for m in meshes]
    # alone: one request at a time
    for i, mid in enumerate(ids):
        srv.wait(srv.submit(mid, states[i], res_alone[i]))
    # in the mix: all requests submitted together
    tickets = [srv.submit(mid, states[i], res_mix[i]) for i, mid in enumerate(ids)]
    for tk in tickets:
        assert srv.wait(tk) >= 0
    for i in range(len(meshes)):
        assert torch.equal(res_alone[i], res_mix[i]), i
    # the resident residual and matrix equal the single-mesh plan results
    for i, (m, mid) in enumerate(zip(meshes, ids)):
        x = torch.from_numpy(np.ascontiguousarray(m.states).reshape(-1)).to(cuda)
        R_alone, y_alone = _alone(fem, cuda, m, x, precision)
        assert torch.equal(res_mix[i], R_alone), i
        o = srv.outputs(mid)
        y = torch.empty_like(x)
        fem.lib.fem_bsr_spmv(m.num_nodes, o["rowp"], o["cols"], o["mat"], x.data_ptr(), y.data_ptr(),
                             torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert torch.equal(y.cpu(), y_alone), i
    if precision == "fp64":
        m = meshes[0]
        rowp, cols = fem.build_bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
        mp = orc.element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols)
        R0, _ = orc.assemble(m, mp, cols.size)
        assert np.abs(res_mix[0].numpy() - R0).max() <= 1e-12 * np.abs(R0).max()
    st = srv.stats()
    assert st["completed"] == 2 * len(meshes)
    # how many requests share a wave depends on timing (the server never waits
    # to fill a wave), so only the bound is fixed
    assert 1 <= st["waves"] <= 2 * len(meshes)
    srv.close()


def test_budget_admission(fem, cuda):
    big = fem.square_mesh(40, 40, 3)
    small = fem.square_mesh(4, 4, 1)
    srv = fem.Server(8 << 20, max_batch=8)  # the 40x40 p=3 mesh needs about 15 MB
    with pytest.raises(fem.FemError) as ei:
        srv.add_mesh(big)
    assert ei.value.status == fem.FEM_ERR_BUDGET
    ids = [srv.add_mesh(small) for _ in range(3)]
    used = srv.stats()["used_bytes"]
    assert 0 < used <= 8 << 20
    srv.remove_mesh(ids[1])
    assert srv.stats()["used_bytes"] < used
    with pytest.raises(fem.FemError):
        srv.remove_mesh(ids[1])
    srv.close()


def test_concurrent_clients(fem, cuda):
    import torch
    meshes = _meshes(fem)[:8]
    srv = fem.Server(8 << 30, max_batch=4)
    ids = [srv.add_mesh(m) for m in meshes]
    ref = []
    for i, m in enumerate(meshes):
        r = torch.empty(m.num_nodes * 2, dtype=torch.float64).pin_memory()
        srv.wait(srv.submit(ids[i], torch.from_numpy(np.ascontiguousarray(m.states)).pin_memory(), r))
        ref.append(r.clone())
    errors = []

    def client(i):
        m = meshes[i]
        st = torch.from_numpy(np.ascontiguousarray(m.states)).pin_memory()
        out = torch.empty(m.num_nodes * 2, dtype=torch.float64).pin_memory()
        for _ in range(5):
            srv.wait(srv.submit(ids[i], st, out))
            if not torch.equal(out, ref[i]):
                errors.append(i)

    threads = [threading.Thread(target=client, args=(i,)) for i in range(len(meshes))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors
    # one request per mesh may be in flight
    st = torch.from_numpy(np.ascontiguousarray(meshes[0].states)).pin_memory()
    tk = srv.submit(ids[0], st)
    with pytest.raises(fem.FemError):
        srv.submit(ids[0], st)
    srv.wait(tk)
    srv.close()


def test_bad_requests_and_abandoned_clients(fem, cuda):
    """A request for an unknown mesh is refused; a client that submits and never
    waits does not hold back the others."""
    import torch
    meshes = _meshes(fem)[:4]
    srv = fem.Server(4 << 30, max_batch=8)
    ids = [srv.add_mesh(m) for m in meshes]
    st = [torch.from_numpy(np.ascontiguousarray(m.states)).pin_memory() for m in meshes]
    with pytest.raises(fem.FemError) as ei:
        srv.submit(99, st[0])
    assert ei.value.status == fem.FEM_ERR_INVALID_ARGUMENT
    srv.submit(ids[0], st[0])  # abandoned: never waited for
    for _ in range(3):
        for i in (1, 2, 3):
            srv.wait(srv.submit(ids[i], st[i]), timeout_ms=20000)
    with pytest.raises(fem.FemError):
        srv.wait(123456789, timeout_ms=10)
    srv.close()
