"""GPU: batched assembly of many meshes of mixed orders (work queues, CUDA graph,
tile autotuner).  Each mesh's result in the batch must equal, bit for bit, its
result assembled alone through its plan, and match the FP64 oracle."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _specs(fem):
    out = []
    for i, spec in enumerate(fem.batch_specs(count=14, lo=2, hi=300, seed=1234)):
        out.append(spec)
    return out


def _setup(fem, cuda, specs):
    import torch
    meshes = [s.build() for s in specs]
    plans = [fem.Plan(m.order, m.num_nodes, m.conn_ptr, m.conn) for m in meshes]
    devs = [fem.DeviceMesh(m, cuda) for m in meshes]
    res = [torch.full((m.num_nodes * 2,), float("nan"), dtype=torch.float64, device=cuda) for m in meshes]
    mat = [torch.full((p.nnzb * 4,), float("nan"), dtype=torch.float64, device=cuda) for p in plans]
    return meshes, plans, devs, res, mat


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_equals_alone_bitwise(fem, orc, cuda, precision):
    import torch
    specs = _specs(fem)
    assert {s.order for s in specs} == {1, 2, 3, 4}
    meshes, plans, devs, res, mat = _setup(fem, cuda, specs)
    batch = fem.Batch(plans)
    for i, (m, d) in enumerate(zip(meshes, devs)):
        batch.bind(i, d.states, d.coords, m.E, m.nu, m.t, res[i], mat[i])
    info = batch.info()
    assert info["elements"] == sum(m.num_elements for m in meshes)
    batch.assemble(precision=precision)
    torch.cuda.synchronize()
    batched = [(r.cpu().numpy().copy(), a.cpu().numpy().copy()) for r, a in zip(res, mat)]
    for i, (m, p, d) in enumerate(zip(meshes, plans, devs)):
        r1 = torch.full_like(res[i], 5.0)
        a1 = torch.full_like(mat[i], 5.0)
        if m.order > 1:
            p.set_layout("colours")  # batches run the colour layout
        p.assemble(d.states, d.coords, m.E, m.nu, m.t, r1, a1, precision=precision)
        torch.cuda.synchronize()
        assert np.array_equal(r1.cpu().numpy(), batched[i][0]), i
        assert np.array_equal(a1.cpu().numpy(), batched[i][1]), i
        if precision == "fp64" and i % 3 == 0:
            rowp, cols = p.pattern()
            mp = orc.element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols)
            R0, A0 = orc.assemble(m, mp, cols.size)
            assert np.abs(batched[i][0] - R0).max() <= 1e-12 * np.abs(R0).max()
            assert np.abs(batched[i][1] - A0).max() <= 1e-12 * np.abs(A0).max()
    batch.close()


def test_batch_tune_capture_replay(fem, cuda):
    import torch
    specs = _specs(fem)
    meshes, plans, devs, res, mat = _setup(fem, cuda, specs)
    batch = fem.Batch(plans)
    for i, (m, d) in enumerate(zip(meshes, devs)):
        batch.bind(i, d.states, d.coords, m.E, m.nu, m.t, res[i], mat[i])
    batch.assemble()
    torch.cuda.synchronize()
    ref = [(r.clone(), a.clone()) for r, a in zip(res, mat)]
    best = batch.tune(reps=2)
    assert best > 0
    info = batch.info()
    assert all(t >= 1 for t in info["tile_batches"])
    # the tuner may pick another FP64 kernel variant per order: equal results
    # within the FP64 tolerance, bit for bit where every order kept its default
    kernels = info["kernels_fp64"]
    exact = kernels == ["rows", "fragment_fp64", "fragment_fp64", "fragment_fp64"]

    def same(x, y):
        if exact:
            return torch.equal(x, y)
        return float((x - y).abs().max()) <= 1e-12 * float(y.abs().max())

    for r, a in zip(res, mat):
        r.fill_(1.0)
        a.fill_(1.0)
    batch.capture()
    secs = batch.replay(timed=True)
    assert secs > 0
    for (r, a), (r0, a0) in zip(zip(res, mat), ref):
        assert same(r, r0) and same(a, a0)
    # a new state is picked up by the graph (the mesh table is read at run time)
    d0 = devs[0]
    d0.states.mul_(2.0)
    batch.replay()
    torch.cuda.synchronize()
    assert torch.allclose(res[0], 2.0 * ref[0][0], rtol=1e-12, atol=0)
    # tiles of one element batch each give the same answer
    batch.set_tiles([1, 1, 1, 1])
    d0.states.mul_(0.5)
    batch.assemble()
    torch.cuda.synchronize()
    for (r, a), (r0, a0) in zip(zip(res, mat), ref):
        assert same(r, r0) and same(a, a0)
    batch.close()


def test_batch_tables_reach_nonblocking_streams(fem, cuda):
    """Tile and mesh tables rebuilt between runs (new tile lengths, the tuner) are in
    place before launches on a non-blocking stream read them: results unchanged."""
    import torch
    specs = _specs(fem)
    meshes, plans, devs, res, mat = _setup(fem, cuda, specs)
    batch = fem.Batch(plans)
    for i, (m, d) in enumerate(zip(meshes, devs)):
        batch.bind(i, d.states, d.coords, m.E, m.nu, m.t, res[i], mat[i])
    batch.assemble()
    torch.cuda.synchronize()
    ref = [(r.clone(), a.clone()) for r, a in zip(res, mat)]
    stream = torch.cuda.Stream(device=cuda)  # created non-blocking
    for tiles in ([1, 1, 1, 1], [256, 64, 16, 4], [4, 1, 64, 16], [16, 16, 16, 16]) * 3:
        batch.set_tiles(tiles)
        for r, a in zip(res, mat):
            r.fill_(float("nan"))
            a.fill_(float("nan"))
        torch.cuda.synchronize()
        batch.assemble(stream=stream.cuda_stream)
        stream.synchronize()
        for (r, a), (r0, a0) in zip(zip(res, mat), ref):
            assert torch.equal(r, r0) and torch.equal(a, a0), tiles
    batch.tune(stream=stream.cuda_stream, reps=1)
    exact = batch.kernels("fp64") == ["rows", "fragment_fp64", "fragment_fp64", "fragment_fp64"]
    batch.assemble(stream=stream.cuda_stream)
    stream.synchronize()
    for (r, a), (r0, a0) in zip(zip(res, mat), ref):
        if exact:
            assert torch.equal(r, r0) and torch.equal(a, a0)
        else:
            assert float((a - a0).abs().max()) <= 1e-12 * float(a0.abs().max())
    batch.close()


VARIANTS = {  # per order: the variants each precision may run
    "fp64": [["rows", "element_fp64"], ["fragment_fp64", "element_fp64"], ["fragment_fp64", "element_fp64"],
             ["fragment_fp64", "element_fp64"]],
    "mixed": [["rows", "element_fp64", "element_fp32"], ["fragment_fp64", "element_fp64", "element_fp32"],
              ["fragment_bf16x6", "fragment_fp64", "element_fp64", "element_fp32"],
              ["element_fp32", "element_tcgen05", "fragment_fp64", "element_fp64"]],
}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_every_kernel_variant(fem, orc, cuda, precision):
    """Every kernel variant the tuner may choose gives the oracle's result: within
    1e-12 normwise for FP64 variants, 1e-6 relative Frobenius for reduced ones."""
    import torch
    specs = _specs(fem)
    meshes, plans, devs, res, mat = _setup(fem, cuda, specs)
    batch = fem.Batch(plans)
    for i, (m, d) in enumerate(zip(meshes, devs)):
        batch.bind(i, d.states, d.coords, m.E, m.nu, m.t, res[i], mat[i])
    refs = []
    for m, p in zip(meshes, plans):
        rowp, cols = p.pattern()
        refs.append(orc.assemble(m, orc.element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols),
                                 cols.size))
    default = [v[0] for v in VARIANTS[precision]]
    if precision == "mixed" and os.environ.get("FEM_ORDER4_MIXED_STIFFNESS") == "tcgen05":
        default[3] = "element_tcgen05"  # the library's order-4 MIXED default follows that switch
    assert batch.kernels(precision) == default
    tiles0 = batch.info()["tile_batches"]
    # each variant with the default tiles and with tiles of one element batch (a
    # group's first batch is then its tile's last: the queue slot is rewritten at once)
    for k, tiles in [(k, t) for k in range(4) for t in (tiles0, [1, 1, 1, 1])]:
        names = [v[min(k, len(v) - 1)] for v in VARIANTS[precision]]
        batch.set_kernels(names, precision)
        batch.set_tiles(tiles)
        assert batch.kernels(precision) == names
        for r, a in zip(res, mat):
            r.fill_(float("nan"))
            a.fill_(float("nan"))
        batch.assemble(precision=precision)
        torch.cuda.synchronize()
        for i, (m, (R0, A0)) in enumerate(zip(meshes, refs)):
            R, A = res[i].cpu().numpy(), mat[i].cpu().numpy()
            reduced = names[m.order - 1] in ("fragment_bf16x6", "element_fp32", "element_tcgen05")
            if names[m.order - 1] in ("element_fp32", "element_tcgen05"):  # FP32 gradients feed the residual too
                assert np.linalg.norm(R - R0) <= 1e-6 * np.linalg.norm(R0), (names, i)
            else:
                assert np.abs(R - R0).max() <= 1e-12 * np.abs(R0).max(), (names, i)
            if reduced:
                assert np.linalg.norm(A - A0) <= 1e-6 * np.linalg.norm(A0), (names, i)
            else:
                assert np.abs(A - A0).max() <= 1e-12 * np.abs(A0).max(), (names, i)
    with pytest.raises(fem.FemError) as ei:
        batch.set_kernels(["fragment_fp64", "rows", "rows", "rows"], precision)
    assert ei.value.status == fem.FEM_ERR_INVALID_ARGUMENT
    if precision == "fp64":
        with pytest.raises(fem.FemError):
            batch.set_kernels(["rows", "element_fp32", "fragment_fp64", "fragment_fp64"], "fp64")
    batch.close()


def test_batch_errors(fem, cuda):
    m = fem.square_mesh(2, 2, 1)
    p = fem.Plan(1, m.num_nodes, m.conn_ptr, m.conn)
    b = fem.Batch([p])
    with pytest.raises(fem.FemError) as ei:
        b.assemble()
    assert ei.value.status == fem.FEM_ERR_INVALID_ARGUMENT  # mesh 0 not bound
    with pytest.raises(fem.FemError):
        b.replay()  # nothing captured
    b.close()
