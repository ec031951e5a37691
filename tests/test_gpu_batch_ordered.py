"""GPU: a batch's colours as one dependency-ordered launch per order
(fem_batch_set_ordered).  A tile waits, bounded, for its mesh's previous colour,
so each block still receives its contributions in colour order: the result must
equal the per-colour launches bit for bit, in every tile length, through a
captured graph, and a wait that is made to run out must end the launch with a
readable count and leave the context usable."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


def _batch(fem, cuda, seed=4321, count=12):
    import torch
    specs = list(fem.batch_specs(count=count, lo=2, hi=300, seed=seed))
    meshes = [s.build() for s in specs]
    plans = [fem.Plan(m.order, m.num_nodes, m.conn_ptr, m.conn) for m in meshes]
    devs = [fem.DeviceMesh(m, cuda) for m in meshes]
    res = [torch.full((m.num_nodes * 2,), float("nan"), dtype=torch.float64, device=cuda) for m in meshes]
    mat = [torch.full((p.nnzb * 4,), float("nan"), dtype=torch.float64, device=cuda) for p in plans]
    batch = fem.Batch(plans)
    for i, (m, d) in enumerate(zip(meshes, devs)):
        batch.bind(i, d.states, d.coords, m.E, m.nu, m.t, res[i], mat[i])
    return meshes, plans, batch, res, mat


def _snapshot(res, mat):
    import torch
    torch.cuda.synchronize()
    return [(r.cpu().numpy().copy(), a.cpu().numpy().copy()) for r, a in zip(res, mat)]


def _clear(res, mat):
    for r, a in zip(res, mat):
        r.fill_(float("nan"))
        a.fill_(float("nan"))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ordered_equals_colour_launches_bitwise(fem, orc, cuda, precision):
    meshes, plans, batch, res, mat = _batch(fem, cuda)
    try:
        assert {m.order for m in meshes} >= {2, 3, 4}
        batch.assemble(precision=precision)
        ref = _snapshot(res, mat)
        launches = batch.info()["launches"]
        batch.set_ordered([0, 1, 1, 1])
        assert batch.ordered() == [0, 1, 1, 1]
        assert batch.info()["launches"] < launches
        for tiles in ([16, 16, 16, 16], [16, 1, 1, 1], [16, 64, 64, 64]):
            batch.set_tiles(tiles)
            _clear(res, mat)
            batch.assemble(precision=precision)
            got = _snapshot(res, mat)
            for i in range(len(meshes)):
                assert np.array_equal(got[i][0], ref[i][0]), (tiles, i)
                assert np.array_equal(got[i][1], ref[i][1]), (tiles, i)
        assert batch.wait_status() == 0
        # through a captured graph, twice
        batch.capture(precision=precision)
        for _ in range(2):
            _clear(res, mat)
            batch.replay()
            got = _snapshot(res, mat)
            for i in range(len(meshes)):
                assert np.array_equal(got[i][0], ref[i][0]), i
                assert np.array_equal(got[i][1], ref[i][1]), i
        if precision == "fp64":
            for i in (1, 4, 7):
                m, p = meshes[i], plans[i]
                rowp, cols = p.pattern()
                mp = orc.element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols)
                R0, A0 = orc.assemble(m, mp, cols.size)
                assert np.abs(got[i][0] - R0).max() <= FP64_TOL * np.abs(R0).max()
                assert np.abs(got[i][1] - A0).max() <= FP64_TOL * np.abs(A0).max()
    finally:
        batch.close()


def test_ordered_bounded_wait_runs_out_and_context_survives(fem, cuda):
    meshes, plans, batch, res, mat = _batch(fem, cuda, seed=97, count=10)
    try:
        order = 3
        assert any(m.order == order and p.num_colours > 1 for m, p in zip(meshes, plans))
        batch.assemble()
        ref = _snapshot(res, mat)
        batch.set_ordered([0, 1, 1, 1])
        # group 0 of order 3: the first order-3 mesh's colour 0, which its colour 1 waits for
        batch.set_schedule_waits(order, wait_limit_ns=20_000_000, stall_group=0)
        batch.assemble()
        assert batch.wait_status() >= 1
        assert batch.wait_status() == 0
        # normal waits again: the same context assembles the same bits
        batch.set_schedule_waits(order, stall_group=-1)
        _clear(res, mat)
        batch.assemble()
        got = _snapshot(res, mat)
        assert batch.wait_status() == 0
        for i in range(len(meshes)):
            assert np.array_equal(got[i][0], ref[i][0]), i
            assert np.array_equal(got[i][1], ref[i][1]), i
    finally:
        batch.close()


def test_ordered_errors(fem, cuda):
    meshes, plans, batch, res, mat = _batch(fem, cuda, seed=98, count=6)
    try:
        with pytest.raises(fem.FemError) as ei:
            batch.set_ordered([1, 0, 0, 0])  # order 1 has no dependency-ordered launch
        assert ei.value.status == fem.FEM_ERR_INVALID_ARGUMENT
        with pytest.raises(fem.FemError) as ei:
            batch.set_schedule_waits(1)
        assert ei.value.status == fem.FEM_ERR_INVALID_ORDER
        batch.set_ordered([0, 1, 1, 1])
        with pytest.raises(fem.FemError) as ei:
            batch.set_schedule_waits(3, stall_group=10 ** 6)
        assert ei.value.status == fem.FEM_ERR_INVALID_ARGUMENT
    finally:
        batch.close()
