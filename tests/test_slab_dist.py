"""The multi-GPU decomposition of one RVE (vpfft_b200/slab.py) on CPU: gloo
ranks in child processes, each holding its x slab of a 5-component field.
Each rank transforms its slab along z (real-to-half-complex) and y, the
all-to-all moves the half spectrum to kz slabs with complete x lines, a
transform along x, a multiplier that depends on the wave vector (the place of
the Green operator) and the inverse transform along x run there, the inverse
all-to-all brings the slabs back, and the inverse y and z transforms finish.
The ranks' pieces, put together, must equal the same pipeline on the whole
array (1e-12), for even and uneven slabs and a rank with an empty slab; the
partial sums all-reduce to the whole-grid sums.  numpy's FFT stands in for
the device line passes here."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _field(dims):
    return np.random.default_rng(3).normal(size=(5,) + dims)


def _multiplier(nx, ny, nh):
    kx = np.arange(nx)[None, None, :]
    ky = np.arange(ny)[None, :, None]
    kz = np.arange(nh)[:, None, None]
    return 1.0 / (1.0 + kx + 2 * ky + 3 * kz)  # [kz][ky][kx]


def _whole(dims):
    nx, ny, nz = dims
    W = _field(dims)
    A = np.fft.rfft(W, axis=3)                     # [c][x][y][kz]
    A = np.fft.fft(A, axis=2)                      # ky
    B = np.transpose(A, (0, 3, 2, 1))              # [c][kz][ky][x]
    B = np.fft.fft(B, axis=3) * _multiplier(nx, ny, nz // 2 + 1)[None]
    B = np.fft.ifft(B, axis=3)
    A = np.transpose(B, (0, 3, 2, 1))
    A = np.fft.ifft(A, axis=2)
    return np.fft.irfft(A, n=nz, axis=3)


def _worker(rank, ws, port, dims, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(ws), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist

    from vpfft_b200 import slab

    dist.init_process_group("gloo", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    try:
        nx, ny, nz = dims
        plan = slab.SlabPlan(nx, ny, nz, ws)
        x0, x1 = plan.x_slabs[rank]
        W = _field(dims)[:, x0:x1]
        A = np.fft.fft(np.fft.rfft(W, axis=3), axis=2)
        B = torch.from_numpy(np.ascontiguousarray(np.transpose(A, (0, 3, 2, 1))))
        Bk = slab.to_x_lines(plan, rank, B).numpy()
        k0, k1 = plan.kz_slabs[rank]
        Bk = np.fft.ifft(np.fft.fft(Bk, axis=3) * _multiplier(nx, ny, plan.nh)[None, k0:k1],
                         axis=3)
        Bx = slab.from_x_lines(plan, rank, torch.from_numpy(np.ascontiguousarray(Bk))).numpy()
        A = np.fft.ifft(np.transpose(Bx, (0, 3, 2, 1)), axis=2)
        out = np.fft.irfft(A, n=nz, axis=3)
        sums = slab.all_reduce_sums(torch.tensor([W.sum(), (W ** 2).sum()])).numpy()
        dist.barrier()
        q.put((rank, x0, x1, out, sums, plan.local_voxels(rank)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("dims,ws", [((8, 6, 10), 2), ((9, 4, 6), 2), ((5, 4, 8), 3),
                                     ((4, 6, 6), 3)])
def test_slab_transposes_match_whole_grid(dims, ws):
    from vpfft_b200 import slab

    plan = slab.SlabPlan(*dims, ws)
    assert sum(plan.local_voxels(r) for r in range(ws)) == int(np.prod(dims))
    assert sum(plan.exchange_elements(s, d) for s in range(ws) for d in range(ws)) == \
        5 * plan.nh * dims[1] * dims[0]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, dims, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(ws))
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    whole = _whole(dims)
    W = _field(dims)
    got = np.zeros_like(whole)
    for rank, x0, x1, out, sums, nv in res:
        got[:, x0:x1] = out
        np.testing.assert_allclose(sums, [W.sum(), (W ** 2).sum()], rtol=1e-12)
    np.testing.assert_allclose(got, whole, rtol=0, atol=1e-12 * np.abs(whole).max())


def test_block_split_is_fftw_default():
    from vpfft_b200 import slab

    assert slab.block_split(16, 3) == [(0, 6), (6, 12), (12, 16)]
    assert slab.block_split(5, 3) == [(0, 2), (2, 4), (4, 5)]
    assert slab.block_split(4, 3) == [(0, 2), (2, 4), (4, 4)]  # an empty rank
