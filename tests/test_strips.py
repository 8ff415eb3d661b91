"""The strip form's host side (no GPU): the column plan and the multi-rank driver.

gbm3d_strip_work runs the library's column planner on the host and reports
the share of the whole image's references a strip matches.  The multi-rank
driver (GBM3D_strips) is run with two gloo ranks on CPU, each computing its
strips through a stand-in strip function (the oracle's whole image, cut to
the strip); the gathered image must equal the one-rank result exactly.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from gbm3d_b200 import api, options, synth
from gbm3d_b200 import distributed as D


def _opts(**kw):
    o = options.resolve_opts({"profile": kw.pop("profile", "default")})
    o.update(kw)
    return o


TUNED = dict(blockSize=8, blockSizeWie=8, refStride=8, refStrideWie=7, matchSpins=[0], matchSpinsWie=[0],
             cycleSpin=1)
DENSE = dict(blockSize=8, blockSizeWie=8, refStride=3, refStrideWie=3)


def test_strip_bounds_partition():
    for n, k in [(10, 3), (4096, 8), (7, 7), (100, 1)]:
        b = D.strip_bounds(n, k)
        assert b[0][0] == 0 and b[-1][1] == n and len(b) == k
        assert all(b[i][1] == b[i + 1][0] and b[i][1] > b[i][0] for i in range(k - 1))
    with pytest.raises(ValueError):
        D.strip_bounds(5, 6)


@pytest.mark.parametrize("kw", [TUNED, DENSE, {}, {"profile": "fast"}, {"Wiener": False}],
                         ids=["tuned", "dense", "default", "fast", "no_wiener"])
def test_strip_work_shares(kw):
    o = _opts(**kw)
    m = n = 1024
    # the whole image: every reference, except those that only reach the
    # padding past column n (the crop drops it)
    whole = api.strip_work(m, n, 0, n, o)
    assert 0.95 <= whole[0] <= 1.0
    assert (0.95 <= whole[1] <= 1.0) if o["Wiener"] else whole[1] == 0.0
    parts = [api.strip_work(m, n, lo, hi, o) for lo, hi in D.strip_bounds(n, 8)]
    for f1, f2 in parts:
        # an eighth of the columns plus its halo: more than an eighth, well under the whole
        assert 0.125 < f1 < 0.6
        assert (0.125 < f2 < 0.4) if o["Wiener"] else f2 == 0.0
    # the eight strips together cover every reference at least once
    assert sum(p[0] for p in parts) >= 1.0
    # a wider strip never matches fewer references
    a = api.strip_work(m, n, 400, 500, o)
    b = api.strip_work(m, n, 380, 520, o)
    assert b[0] >= a[0] and b[1] >= a[1]


def test_strip_work_rejects_bad_columns():
    o = _opts(**TUNED)
    for lo, hi in [(5, 5), (-1, 3), (0, 65)]:
        with pytest.raises(Exception):
            api.strip_work(64, 64, lo, hi, o)


def _oracle_strip(I, sigma, o, lo, hi):
    from oracle import oracle as O
    U, _ = O.GBM3D(I, sigma, o, prec=32)
    return U[:, lo:hi]


def _rank_main(rank, world, port, noisy, sigma, strips, outdir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from oracle import oracle as O
    O.set_threads(2)
    U = D.GBM3D_strips(noisy, sigma, _opts(**TUNED), strips=strips, strip_fn=_oracle_strip)
    np.save(os.path.join(outdir, f"U{rank}_{strips}.npy"), U)
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("strips", [2, 3])
def test_two_rank_strips_match_one_rank(tmp_path, strips):
    from oracle import oracle as O
    clean, noisy = synth.noisy_image(64, 90, 25.0, seed=5)
    U1, _ = O.GBM3D(noisy, 25.0, _opts(**TUNED), prec=32)
    assert options.myPSNR(clean, U1, 255) > options.myPSNR(clean, noisy, 255) + 3
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, noisy, 25.0, strips, str(tmp_path)))
             for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=600)
        assert p.exitcode == 0
    for r in range(2):
        assert np.array_equal(np.load(tmp_path / f"U{r}_{strips}.npy"), U1)
