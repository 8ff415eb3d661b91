"""tcgen05 building blocks: the operand / accumulator layouts of csrc/tc.cuh.

One 128 x 256 x 64 bf16 GEMM through gbm3d_tc_selfcheck against the exact
product of the same bf16 values (fp32 accumulation: relative error ~1e-6).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bf16(x):
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return u.astype(np.uint16)


def _f32(b):
    return (b.astype(np.uint32) << 16).view(np.float32)


@pytest.mark.parametrize("seed", [0, 1])
def test_tcgen05_gemm_layouts(gpu, seed):
    from gbm3d_b200._lib import context, lib
    rng = np.random.default_rng(seed)
    A = _bf16(rng.normal(0, 1, (128, 64)))
    B = _bf16(rng.normal(0, 1, (256, 64)))
    out = np.zeros((128, 256), dtype=np.float32)
    ctx = context()
    ctx.check(lib().gbm3d_tc_selfcheck(ctx.h, A.ctypes.data_as(C.c_void_p), B.ctypes.data_as(C.c_void_p),
                                       out.ctypes.data_as(C.c_void_p)))
    ref = _f32(A).astype(np.float64) @ _f32(B).astype(np.float64).T
    err = np.abs(out - ref).max()
    assert err < 1e-4 * np.abs(ref).max(), f"max error {err}"


@pytest.mark.parametrize("mn_major", [0, 1])
def test_tcgen05_gemm_operand_majors(gpu, mn_major):
    """K-major and MN-major operand staging give the same exact product (mode 1:
    the descriptor offsets the pilot's weight gradient uses)."""
    from gbm3d_b200._lib import context, lib
    rng = np.random.default_rng(5 + mn_major)
    A = _bf16(rng.normal(0, 1, (128, 64)))
    B = _bf16(rng.normal(0, 1, (256, 64)))
    out = np.zeros((128, 256), dtype=np.float32)
    ctx = context()
    ctx.check(lib().gbm3d_tc_selfcheck_layout(ctx.h, mn_major, A.ctypes.data_as(C.c_void_p),
                                              B.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p)))
    ref = _f32(A).astype(np.float64) @ _f32(B).astype(np.float64).T
    err = np.abs(out - ref).max()
    assert err < 1e-4 * np.abs(ref).max(), f"max error {err}"


def test_tcgen05_mn_major_offset_reading(gpu):
    """Which reading of the MN-major descriptor offsets the hardware follows:
    exactly one of the two gives the product (reported; mode 1 must be it)."""
    from gbm3d_b200._lib import context, lib
    rng = np.random.default_rng(9)
    A = _bf16(rng.normal(0, 1, (128, 64)))
    B = _bf16(rng.normal(0, 1, (256, 64)))
    ref = _f32(A).astype(np.float64) @ _f32(B).astype(np.float64).T
    ctx = context()
    errs = {}
    for mode in (1, 2):
        out = np.zeros((128, 256), dtype=np.float32)
        ctx.check(lib().gbm3d_tc_selfcheck_layout(ctx.h, mode, A.ctypes.data_as(C.c_void_p),
                                                  B.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p)))
        errs[mode] = float(np.abs(out - ref).max() / np.abs(ref).max())
    print(f"MN-major relative error: leading offset = K stride {errs[1]:.2e}, = MN stride {errs[2]:.2e}")
    assert errs[1] < 1e-4
