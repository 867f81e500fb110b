"""Cell-level transforms (local_map_to_global.cu, cell_broadcast.cu, cell_reduce.cu): the host path
against numpy restatements of the reference loops (CPU), and the device kernels against the host
path (GPU)."""

import numpy as np
import pytest

N = 3 * 64 * 64


def np_broadcast(src, index_map):
    # cell_broadcast.cu:24-35
    return np.concatenate([src[j * N:(j + 1) * N] for j in index_map]) if len(index_map) else np.zeros(0, src.dtype)


def np_reduce(ndst, src, index_map):
    # cell_reduce.cu:27-40
    dst = np.zeros(ndst, src.dtype)
    for i, j in enumerate(index_map):
        dst[j * N:(j + 1) * N] += src[i * N:(i + 1) * N]
    return dst


@pytest.fixture(scope="module")
def m():
    import gpu_mm_b200
    return gpu_mm_b200.gpu_mm_pybind11


def test_cell_broadcast_reduce_host(m):
    rng = np.random.default_rng(0)
    src = rng.standard_normal(5 * N).astype(np.float32)
    im = np.array([3, 0, 3, 4], dtype=np.int64)
    dst = np.zeros(4 * N, np.float32)
    m.cell_broadcast(dst, src, im)
    np.testing.assert_array_equal(dst, np_broadcast(src, im))
    red = np.full(6 * N, 7.0, np.float32)
    src2 = rng.standard_normal(4 * N).astype(np.float32)
    m.cell_reduce(red, src2, im)
    np.testing.assert_array_equal(red, np_reduce(6 * N, src2, im))
    with pytest.raises(RuntimeError):
        m.cell_broadcast(dst, src, np.array([0, 1, 2, 5], dtype=np.int64))
    with pytest.raises(RuntimeError):
        m.cell_reduce(red, src2, np.array([0, 1, 2, 6], dtype=np.int64))


@pytest.mark.gpu
def test_local_map_to_global_host(m):
    """(LocalPixelization keeps a device copy of cell_offsets, so this needs a GPU.)"""
    import gpu_mm_b200 as g
    rng = np.random.default_rng(1)
    ny, nx = 192, 320
    cells = [(0, 1), (2, 4), (1, 0)]
    lp = g.LocalPixelization.make_cells(ny, nx, cells)
    arr = rng.standard_normal(3 * lp.npix).astype(np.float32)
    glob = g.LocalMap(lp, arr).to_global()
    want = np.zeros((3, ny, nx), np.float32)
    for k, (cy, cx) in enumerate(cells):
        off = int(np.asarray(lp.cell_offsets_cpu).reshape(-1)[cy * ((nx + 63) // 64) + cx])
        for p in range(3):
            for iy in range(64):
                want[p, 64 * cy + iy, 64 * cx:64 * cx + 64] = arr[off + p * lp.polstride + iy * lp.ystride:
                                                                 off + p * lp.polstride + iy * lp.ystride + 64]
    np.testing.assert_array_equal(glob, want)


@pytest.mark.gpu
def test_cells_device_match_host(m):
    import torch
    import gpu_mm_b200 as g
    rng = np.random.default_rng(2)
    src = rng.standard_normal(9 * N).astype(np.float32)
    im = rng.integers(0, 9, 20).astype(np.int64)
    dst_h = np.zeros(20 * N, np.float32)
    m.cell_broadcast(dst_h, src, im)
    dst_d = torch.zeros(20 * N, device="cuda")
    m.cell_broadcast(dst_d, torch.from_numpy(src).cuda(), torch.from_numpy(im).cuda())
    np.testing.assert_array_equal(dst_d.cpu().numpy(), dst_h)
    src2 = rng.standard_normal(20 * N).astype(np.float32)
    red_h = np.zeros(9 * N, np.float32)
    m.cell_reduce(red_h, src2, im)
    red_d = torch.full((9 * N,), 3.0, device="cuda")
    m.cell_reduce(red_d, torch.from_numpy(src2).cuda(), torch.from_numpy(im).cuda())
    np.testing.assert_allclose(red_d.cpu().numpy(), red_h, rtol=1e-6, atol=1e-6)
    with pytest.raises(RuntimeError):
        m.cell_broadcast(dst_d, torch.from_numpy(src).cuda(), torch.tensor([0, 9] + [0] * 18, device="cuda"))
    # local map -> global on the device
    ny, nx = 200, 300
    lp = g.LocalPixelization.make_cells(ny, nx, [(0, 0), (3, 4), (1, 2), (2, 0)])
    arr = torch.from_numpy(rng.standard_normal(3 * lp.npix).astype(np.float32)).cuda()
    lm = g.LocalMap(lp, arr)
    np.testing.assert_array_equal(lm.to_global(on_device=True).cpu().numpy(), lm.to_global())
