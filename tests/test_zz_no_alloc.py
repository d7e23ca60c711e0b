"""pdgpu_build_neighbors_noalloc: the peridynamic neighbour lists built with
no device allocation, for hosts whose device memory belongs to another
allocator, against the allocating build of the same library
(pdgpu_build_pd_neighbors, whose sets tests/test_gpu_setup_parity.py ties to
the reference's kd-tree search).  Both sort each row by node index, so rows
must be equal.  Inputs outside the entry point's limits (a sparse domain
that forces the coarse search grid, a node with more than 1024 neighbours,
a stream that is capturing) are checked against a brute-force search or
against the documented error codes.

Device buffers are allocated here by torch; the entry point itself only uses
the caller's buffers and its static scratch array.  Named so that pytest
collects it after every other file: it must pass both alone in a fresh
process and after the other GPU tests.
"""
import ctypes

import numpy as np
import pytest

from peridem_b200 import scene as scn

R = 1e-3
MAX_NODES = 1 << 18
PDGPU_ERR_ARG, PDGPU_ERR_OVERFLOW, PDGPU_ERR_STATE = -1, -4, -6   # codes of include/pdgpu.h


def _call(x, pt, hz, n, dim, rowptr, col, cap, stream=None):
    from peridem_b200 import api
    L = api.lib()
    nb = ctypes.c_int64(-1)
    err = ctypes.create_string_buffer(256)
    rc = L.pdgpu_build_neighbors_noalloc(x, pt, hz, n, dim, rowptr, col, cap, ctypes.byref(nb),
                                         stream, err, len(err))
    return rc, nb.value, err.value.decode()


def _noalloc(sc, calls=2):
    """Run the allocation-free build `calls` times in a row on the scene's
    reference positions; return the (rowptr, col) of every call."""
    import torch
    dev = torch.device("cuda:0")
    N = sc.n_nodes
    x = torch.as_tensor(np.ascontiguousarray(sc.xref, dtype=np.float64), device=dev)
    pt = torch.as_tensor(sc.ptid.astype(np.int32), device=dev)          # uint32 bits
    hz = torch.as_tensor(np.asarray(sc.p_horizon, dtype=np.float64), device=dev)
    rowptr = torch.empty(N + 1, dtype=torch.int64, device=dev)          # uint64 bits
    stream = torch.cuda.current_stream(dev).cuda_stream
    # size query first (col = NULL), then the build
    rc, nb, msg = _call(x.data_ptr(), pt.data_ptr(), hz.data_ptr(), N, sc.dim, rowptr.data_ptr(),
                        None, 0, stream)
    assert rc == 0, msg
    col = torch.full((nb,), -1, dtype=torch.int32, device=dev)
    out = []
    for _ in range(calls):
        rowptr.fill_(-1)
        col.fill_(-1)
        rc, nb2, msg = _call(x.data_ptr(), pt.data_ptr(), hz.data_ptr(), N, sc.dim,
                             rowptr.data_ptr(), col.data_ptr(), nb, stream)
        assert rc == 0, msg
        assert nb2 == nb
        torch.cuda.synchronize()
        out.append((rowptr.cpu().numpy().view(np.uint64).copy(),
                     col.cpu().numpy().view(np.uint32).astype(np.uint64)))
    return out


def _device_inputs(x, pt, hz):
    import torch
    dev = torch.device("cuda:0")
    return (torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64), device=dev),
            torch.as_tensor(np.asarray(pt, dtype=np.int32), device=dev),
            torch.as_tensor(np.asarray(hz, dtype=np.float64), device=dev))


def _brute(x, pt, hz):
    """Rows of the strict squared-distance search, summed in the kd-tree's
    order (dims 0, 1, 2 of query minus point), ascending."""
    n = len(x)
    rows = []
    for i in range(n):
        d = (x[i, 0] - x[:, 0]) * (x[i, 0] - x[:, 0])
        d = d + (x[i, 1] - x[:, 1]) * (x[i, 1] - x[:, 1])
        d = d + (x[i, 2] - x[:, 2]) * (x[i, 2] - x[:, 2])
        r = hz[pt[i]]
        hit = (d < r * r) & (pt == pt[i])
        hit[i] = False
        rows.append(np.nonzero(hit)[0])
    rp = np.zeros(n + 1, dtype=np.uint64)
    rp[1:] = np.cumsum([len(r) for r in rows])
    return rp, np.concatenate(rows).astype(np.uint64)


def _allocating(sc):
    from peridem_b200.model import GpuDEMModel
    m = GpuDEMModel(sc, build_neighbors=True, compute_mx=True)
    try:
        return m.pd_neighbors()
    finally:
        m.close()


def _scenes():
    h = R / 8
    yield "compressive_2d", scn.build_scene(scn.compressive_2d(
        n_particles=40, r_range=(R, 1.3 * R), h_div=8, width=14e-3, seed=11, gap=1.02 * h,
        wall_speed=-2.0, nt=10))
    yield "column_3d", scn.build_scene(scn.column_3d(
        n_spheres=3, median_r=R, sigma=0.0, h_div=5, box=(3e-3, 3e-3, 8e-3), seed=2,
        material="PDState", piston_speed=-2.0, nt=10))


@pytest.mark.gpu
def test_noalloc_matches_allocating_build_twice_in_a_row():
    for name, sc in _scenes():
        assert sc.n_nodes <= MAX_NODES
        rp_ref, col_ref = _allocating(sc)
        runs = _noalloc(sc, calls=2)
        for k, (rp, col) in enumerate(runs):
            assert np.array_equal(rp, rp_ref), f"{name}: row offsets differ on call {k + 1}"
            assert np.array_equal(col, col_ref), f"{name}: columns differ on call {k + 1}"
        print(f"{name}: {sc.n_nodes} nodes, {len(col_ref)} bonds, identical on both calls")


@pytest.mark.gpu
def test_noalloc_reports_short_column_buffer():
    import torch
    _, sc = next(_scenes())
    dev = torch.device("cuda:0")
    N = sc.n_nodes
    x = torch.as_tensor(np.ascontiguousarray(sc.xref, dtype=np.float64), device=dev)
    pt = torch.as_tensor(sc.ptid.astype(np.int32), device=dev)
    hz = torch.as_tensor(np.asarray(sc.p_horizon, dtype=np.float64), device=dev)
    rowptr = torch.empty(N + 1, dtype=torch.int64, device=dev)
    col = torch.empty(16, dtype=torch.int32, device=dev)
    rc, nb, msg = _call(x.data_ptr(), pt.data_ptr(), hz.data_ptr(), N, sc.dim, rowptr.data_ptr(),
                        col.data_ptr(), 16, None)
    assert rc == PDGPU_ERR_OVERFLOW and nb > 16 and "neighbours" in msg


@pytest.mark.gpu
def test_noalloc_coarse_grid_of_a_sparse_domain_matches_brute_force():
    """Two clusters 2e4 horizons apart: the horizon-sized grid would need
    ~4e8 cells, so the build coarsens its cells until they fit the scratch
    array; the sets must not change."""
    import torch
    rng = np.random.default_rng(7)
    h = 1e-4
    a = np.stack([rng.uniform(0, 20 * h, 300), rng.uniform(0, 20 * h, 300), np.zeros(300)], 1)
    b = a + np.array([2e4 * 3 * h, 1e4 * 3 * h, 0.0])
    x = np.concatenate([a, b])
    pt = np.repeat(np.arange(2), 300)
    hz = np.array([3 * h, 3 * h])
    rp_ref, col_ref = _brute(x, pt, hz)
    xd, ptd, hzd = _device_inputs(x, pt, hz)
    N = len(x)
    rowptr = torch.empty(N + 1, dtype=torch.int64, device=xd.device)
    rc, nb, msg = _call(xd.data_ptr(), ptd.data_ptr(), hzd.data_ptr(), N, 2, rowptr.data_ptr(), None, 0)
    assert rc == 0, msg
    col = torch.full((nb,), -1, dtype=torch.int32, device=xd.device)
    for k in range(2):
        rc, nb2, msg = _call(xd.data_ptr(), ptd.data_ptr(), hzd.data_ptr(), N, 2, rowptr.data_ptr(),
                             col.data_ptr(), nb)
        assert rc == 0, msg
        torch.cuda.synchronize()
        assert np.array_equal(rowptr.cpu().numpy().view(np.uint64), rp_ref), f"rows differ on call {k + 1}"
        assert np.array_equal(col.cpu().numpy().view(np.uint32).astype(np.uint64), col_ref), \
            f"columns differ on call {k + 1}"


@pytest.mark.gpu
def test_noalloc_size_query_refuses_rows_longer_than_it_sorts():
    """A 40 x 40 grid with a horizon of 30 spacings: inner nodes have ~2800
    neighbours; the size query already reports PDGPU_ERR_OVERFLOW."""
    import torch
    h = 1e-4
    g = np.arange(40) * h
    X, Y = np.meshgrid(g, g, indexing="ij")
    x = np.stack([X.ravel(), Y.ravel(), np.zeros(X.size)], 1)
    pt = np.zeros(len(x), dtype=np.int64)
    hz = np.array([30 * h])
    xd, ptd, hzd = _device_inputs(x, pt, hz)
    rowptr = torch.empty(len(x) + 1, dtype=torch.int64, device=xd.device)
    rc, nb, msg = _call(xd.data_ptr(), ptd.data_ptr(), hzd.data_ptr(), len(x), 2, rowptr.data_ptr(),
                        None, 0)
    assert rc == PDGPU_ERR_OVERFLOW, (rc, msg)
    assert "1024" in msg


@pytest.mark.gpu
def test_noalloc_refuses_a_capturing_stream():
    """The call blocks the host, so it must refuse to run inside a capture
    instead of breaking it."""
    import torch
    _, sc = next(_scenes())
    xd, ptd, hzd = _device_inputs(sc.xref, sc.ptid.astype(np.int64), sc.p_horizon)
    N = sc.n_nodes
    rowptr = torch.empty(N + 1, dtype=torch.int64, device=xd.device)
    side = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    scratch = torch.zeros(4, device=xd.device)
    with torch.cuda.graph(g, stream=side):
        scratch.add_(1.0)
        rc, _, msg = _call(xd.data_ptr(), ptd.data_ptr(), hzd.data_ptr(), N, sc.dim, rowptr.data_ptr(),
                           None, 0, side.cuda_stream)
    del g
    assert rc == PDGPU_ERR_STATE, (rc, msg)
    assert "capture" in msg


def test_noalloc_rejects_too_many_nodes_before_touching_the_device():
    # the size check comes before any CUDA call, so this runs without a GPU;
    # the pointers are never dereferenced
    fake = 0x1000
    rc, _, msg = _call(fake, fake, fake, MAX_NODES + 1, 3, fake, fake, 1, None)
    assert rc == PDGPU_ERR_ARG
    assert "262144" in msg and "maximum" in msg
