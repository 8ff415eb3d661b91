"""gbm3d_matchBlocks_noalloc against gbm3d_matchBlocksCPU, through the C ABI.

The allocation-free entry point serves callers that may not allocate device
memory while they run (servers and video pipelines that reserve all GPU
memory at start-up, hosts whose allocator owns every device buffer).  Its
scratch is a fixed device array shared by all calls, so this test makes two
calls in a row on different images and checks each against the allocating
entry point: identical match sets and counts.  The test allocates its own
input and output buffers with torch; the entry point itself allocates none.
This file sorts last so that a stop-at-first-failure run has already run
every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_matching_matches_allocating_entry_point(gpu):
    import torch

    from gbm3d_b200 import _lib, api, options, synth

    L = _lib.lib()
    opts = options.resolve_opts({"profile": "default"})
    co = api.c_opts(opts)
    d, K = opts["blockSize"], opts["numMax"]
    for call, (m, n, sigma, seed) in enumerate([(160, 128, 25.0, 31), (96, 144, 10.0, 32)]):
        _, noisy = synth.noisy_image(m, n, sigma, seed=seed)
        img32 = np.asfortranarray(noisy.astype(np.float32))
        M, N = m // d, n // d
        dI = torch.from_numpy(img32.ravel(order="F")).cuda()
        dS = torch.zeros(K * M * N, dtype=torch.int32, device="cuda")
        dc = torch.zeros(M * N, dtype=torch.int32, device="cuda")
        rc = L.gbm3d_matchBlocks_noalloc(C.c_void_p(dI.data_ptr()), m, n, sigma, C.byref(co),
                                        C.c_void_p(dS.data_ptr()), C.c_void_p(dc.data_ptr()), None)
        assert rc == 0, f"call {call}: rc={rc}"
        torch.cuda.synchronize()
        S = dS.cpu().numpy().view(np.uint32).reshape((K, M, N), order="F")
        cnt = dc.cpu().numpy().reshape((M, N), order="F")
        # the allocating entry point on the same single-precision image
        Sref, _ = api.matchBlocksCPU(img32.astype(np.float64), sigma, opts)
        assert np.array_equal(S, np.asarray(Sref)), f"call {call}: match sets differ"
        assert np.array_equal(cnt, Sref.count), f"call {call}: counts differ"


def test_noalloc_rejects_images_beyond_the_scratch(gpu):
    from gbm3d_b200 import _lib, api, options

    L = _lib.lib()
    co = api.c_opts(options.resolve_opts({"profile": "default"}))
    # sizes only: the check happens before any pointer is used
    rc = L.gbm3d_matchBlocks_noalloc(C.c_void_p(16), 4096, 4096, 25.0, C.byref(co), C.c_void_p(16), None, None)
    assert rc == 6  # GBM3D_ERR_TOO_LARGE
