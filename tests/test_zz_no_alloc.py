"""pdgpu_build_neighbors_noalloc: the peridynamic neighbour lists built with
no device allocation, against the allocating build of the same library
(pdgpu_build_pd_neighbors, whose sets the parity tests tie to the reference's
kd-tree search).  Both sort each row by node index, so rows must be equal.

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
PDGPU_ERR_ARG, PDGPU_ERR_OVERFLOW = -1, -4   # codes of include/pdgpu.h


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


def test_noalloc_rejects_too_many_nodes_before_touching_the_device():
    # the size check comes before any CUDA call, so this runs without a GPU;
    # the pointers are never dereferenced
    fake = 0x1000
    rc, _, msg = _call(fake, fake, fake, MAX_NODES + 1, 3, fake, fake, 1, None)
    assert rc == PDGPU_ERR_ARG
    assert "262144" in msg and "maximum" in msg
