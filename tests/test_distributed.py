"""GBM3D_distributed tiling, stitching and its multi-rank sharding.

The tiling and ramp windows are checked against the reference's rules
(getBM3D_distribution.m:10-48, makeInterpWindow.m:8-13).  Sharding is checked
on CPU with two gloo ranks: each rank denoises its share of the tiles with the
CPU oracle as backend, the results are all-gathered, and both ranks must
produce exactly the one-rank result.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from gbm3d_b200 import distributed as D
from gbm3d_b200 import options, synth


@pytest.mark.parametrize("m,n,k", [(300, 290, 16), (512, 600, 16), (4096, 4096, 16), (280, 300, 8), (700, 333, 32)])
def test_distribution_covers_and_aligns(m, n, k):
    R, d0, _ = D.getBM3D_distribution(m, n, [0, 4], k)
    assert d0 == 256 + k
    cover = np.zeros((m, n), dtype=int)
    for r1, r2, r3, r4, s in R:
        assert 1 <= r1 <= r2 <= m and 1 <= r3 <= r4 <= n
        assert (r2 - r1 + 1) % k == 0 and (r4 - r3 + 1) % k == 0  # tiles hold whole reference blocks
        assert (r2 - r1 + 1) >= 2 * k and (r4 - r3 + 1) >= 2 * k
        cover[r1 - 1:r2, r3 - 1:r4] += 1
    assert cover.min() >= 2  # every pixel in at least one tile per spin
    assert sorted(set(R[:, 4].tolist())) == [0, 4]


def test_distribution_known_rows():
    # 300 x 300, k=16: 2x2 tiles; the second row/column tiles are pulled back to
    # start at 253 so that their length (48) is a multiple of 16.
    R, _, _ = D.getBM3D_distribution(300, 300, [0], 16)
    assert R.tolist() == [[1, 272, 1, 272, 0], [1, 272, 253, 300, 0], [253, 300, 1, 272, 0],
                          [253, 300, 253, 300, 0]]


def test_interp_window():
    w = D.makeInterpWindow(40, 36, 8)
    ramp = np.linspace(0.01, 1, 8)
    assert np.allclose(w[8:32, 0], ramp[0]) and np.allclose(w[0, 8:28], ramp[0])
    assert np.allclose(w[20, :8], ramp) and np.allclose(w[20, -8:], ramp[::-1])
    assert np.allclose(w[10:30, 10:26], 1.0)
    assert np.isclose(w[0, 0], ramp[0] ** 2)


def oracle_backend():
    from oracle import oracle as O

    def step1(I, sigma, tau, opts):
        S, V, cnt = O.matchBlocksCPU(I, sigma, opts, prec=32)
        return O.denoiseAndAggregateGPU(V, S, tau, opts, cnt=cnt, prec=32)

    def step2(P, I, sigma, opts):
        S, V1, V2 = O.matchBlocksWie(P, I, sigma, opts, prec=32)
        return O.denoiseAndAggregateWieFast(V1, V2, S, sigma, opts, prec=32)

    return D.Backend(step1, step2)


def _rank_main(rank, world, port, noisy, sigma, outdir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from oracle import oracle as O
    O.set_threads(2)
    U, out = D.GBM3D_distributed(noisy, sigma, {"profile": "default"}, backend=oracle_backend())
    np.save(os.path.join(outdir, f"U{rank}.npy"), U)
    np.save(os.path.join(outdir, f"U2_{rank}.npy"), out["U2"])
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_sharding_matches_one_rank(tmp_path):
    clean, noisy = synth.noisy_image(290, 300, 25.0, seed=41)
    U1, out1 = D.GBM3D_distributed(noisy, 25.0, {"profile": "default"}, backend=oracle_backend())
    assert options.myPSNR(clean, U1, 255) > options.myPSNR(clean, noisy, 255) + 5
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, noisy, 25.0, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=600)
        assert p.exitcode == 0
    for r in range(2):
        assert np.array_equal(np.load(tmp_path / f"U{r}.npy"), U1)
        assert np.array_equal(np.load(tmp_path / f"U2_{r}.npy"), out1["U2"])


def test_small_image_falls_back_to_gbm3d(monkeypatch):
    called = {}

    def fake(I, sigma, o):
        called["yes"] = True
        return I, {}
    import gbm3d_b200.api as api
    monkeypatch.setattr(api, "GBM3D", fake)
    D.GBM3D_distributed(np.zeros((200, 300)), 25.0)
    assert called.get("yes")
