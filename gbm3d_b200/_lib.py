"""ctypes binding of libgbm3d.so (include/gbm3d.h).

The library is the product: there is no CPU fallback.  If the shared library
is missing, or no CUDA device can be opened, every compute call raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgbm3d.so")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "gbm3d.h")

GBM3D_OK = 0
ERRORS = {1: "invalid argument", 2: "CUDA error", 3: "out of device memory",
          4: "non-finite input", 5: "unsupported option", 6: "image too large for the fixed scratch"}


class GBM3DError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"gbm3d error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class gbm3d_opts(C.Structure):
    _fields_ = [
        ("numMax", C.c_int), ("numMin", C.c_int),
        ("blockSize", C.c_int), ("blockSizeWie", C.c_int), ("matchSize", C.c_int), ("refStride", C.c_int),
        ("levels", C.c_int), ("cycleSpin", C.c_int), ("tauMode", C.c_int),
        ("Wiener", C.c_int), ("filtType", C.c_int),
        ("nMatchSpins", C.c_int), ("matchSpins", C.c_int * 8),
        ("nMatchSpinsWie", C.c_int), ("matchSpinsWie", C.c_int * 8),
        ("staleWeights", C.c_int), ("refStrideWie", C.c_int), ("wavelet", C.c_int),
        ("form", C.c_int), ("videoFrames", C.c_int),
    ]


class gbm3d_filters(C.Structure):
    _fields_ = [
        ("len_xy", C.c_int),
        ("a_lo_xy", C.c_double * 16), ("a_hi_xy", C.c_double * 16),
        ("s_lo_xy", C.c_double * 16), ("s_hi_xy", C.c_double * 16),
        ("len_z", C.c_int),
        ("a_lo_z", C.c_double * 16), ("a_hi_z", C.c_double * 16),
        ("s_lo_z", C.c_double * 16), ("s_hi_z", C.c_double * 16),
    ]


class gbm3d_mixed_batch(C.Structure):
    _fields_ = [
        ("n_grey", C.c_int), ("grey", C.c_void_p), ("grey_m", C.c_void_p), ("grey_n", C.c_void_p),
        ("grey_sigma", C.c_void_p), ("grey_out", C.c_void_p),
        ("n_rgb", C.c_int), ("rgb", C.c_void_p), ("rgb_m", C.c_void_p), ("rgb_n", C.c_void_p),
        ("rgb_sigma", C.c_void_p), ("rgb_out", C.c_void_p),
        ("video", C.c_void_p), ("video_m", C.c_int), ("video_n", C.c_int), ("video_frames", C.c_int),
        ("video_sigma", C.c_double), ("video_out", C.c_void_p),
        ("grey_opts", C.c_void_p), ("rgb_opts", C.c_void_p),
    ]


_P = C.c_void_p
_SIGS = {
    "gbm3d_version": (C.c_int, []),
    "gbm3d_ctx_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "gbm3d_ctx_destroy": (None, [_P]),
    "gbm3d_ctx_set_stream": (C.c_int, [_P, _P]),
    "gbm3d_last_error": (C.c_char_p, [_P]),
    "gbm3d_default_opts": (None, [C.c_char_p, C.POINTER(gbm3d_opts)]),
    "gbm3d_get_tau": (None, [C.c_int, C.c_int, _P]),
    "gbm3d_bior_filters": (None, [C.POINTER(gbm3d_filters)]),
    "gbm3d_matchBlocksCPU": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_double, C.POINTER(gbm3d_opts), _P, _P, _P]),
    "gbm3d_matchBlocksGPU": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_double, C.POINTER(gbm3d_opts), _P, _P]),
    "gbm3d_denoiseAndAggregateGPU": (C.c_int, [_P, _P, _P, _P, C.c_int, C.c_int, _P, C.POINTER(gbm3d_filters),
                                               C.POINTER(gbm3d_opts), _P, _P]),
    "gbm3d_matchBlocksWie": (C.c_int, [_P, _P, _P, C.c_int, C.c_int, C.c_double, C.POINTER(gbm3d_opts), _P, _P, _P]),
    "gbm3d_denoiseAndAggregateWieFast": (C.c_int, [_P, _P, _P, _P, C.c_int, C.c_int, _P, C.c_int,
                                                   C.POINTER(gbm3d_opts), _P, _P]),
    "gbm3d_denoiseAndAggregateWie": (C.c_int, [_P, _P, _P, _P, C.c_int, C.c_int, C.c_double,
                                               C.POINTER(gbm3d_opts), _P, _P]),
    "gbm3d_denoise": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_double, C.POINTER(gbm3d_opts), _P, _P]),
    "gbm3d_denoise_device": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_double, C.POINTER(gbm3d_opts), _P, _P]),
    "gbm3d_denoise_async": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_double, C.POINTER(gbm3d_opts), _P]),
    "gbm3d_denoise_strip_device": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_double, C.POINTER(gbm3d_opts), C.c_int,
                                             C.c_int, _P]),
    "gbm3d_strip_work": (C.c_int, [C.POINTER(gbm3d_opts), C.c_int, C.c_int, C.c_int, C.c_int, _P]),
    "gbm3d_ctx_enable_timing": (C.c_int, [_P, C.c_int]),
    "gbm3d_ctx_set_tc_wait": (C.c_int, [_P, C.c_longlong]),
    "gbm3d_ctx_set_lanes": (C.c_int, [_P, C.c_int]),
    "gbm3d_ctx_tc_stats": (C.c_int, [_P, C.c_int, _P]),
    "gbm3d_stage_times": (C.c_int, [_P, _P, C.c_int]),
    "gbm3d_last_launch_count": (C.c_int, [_P]),
    "gbm3d_kernel_time": (C.c_int, [_P, C.c_char_p, _P]),
    "gbm3d_filters_from_bank": (C.c_int, [_P, _P, C.c_int, C.c_int, C.POINTER(gbm3d_filters)]),
    "gbm3d_tc_selfcheck": (C.c_int, [_P, _P, _P, _P]),
    "gbm3d_tc_selfcheck_layout": (C.c_int, [_P, C.c_int, _P, _P, _P]),
    "gbm3d_tiles_device": (C.c_int, [_P, _P, _P, C.c_int, C.c_int, C.c_double, _P, C.POINTER(gbm3d_opts), _P,
                                     C.c_int, C.c_int, _P]),
    "gbm3d_tiles_stitch_device": (C.c_int, [_P, _P, _P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _P, _P]),
    "gbm3d_ctx_synchronize": (C.c_int, [_P]),
    "gbm3d_denoise_rgb_device": (C.c_int, [_P, _P, _P, _P, C.c_int, C.c_int, C.c_double, C.POINTER(gbm3d_opts),
                                           _P, _P, _P]),
    "gbm3d_vbm3d_device": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int, C.c_double, C.POINTER(gbm3d_opts), _P]),
    "gbm3d_matchBlocksV": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int, C.POINTER(gbm3d_opts), _P, _P]),
    "gbm3d_denoiseAndAggregateV": (C.c_int, [_P, _P, _P, C.c_int, C.c_int, C.c_int, _P, C.POINTER(gbm3d_filters),
                                             C.POINTER(gbm3d_opts), _P, _P]),
    "gbm3d_denoise_batch": (C.c_int, [_P, C.c_int, _P, _P, _P, _P, C.POINTER(gbm3d_opts), _P, C.c_int]),
    "gbm3d_denoise_mixed": (C.c_int, [_P, C.POINTER(gbm3d_mixed_batch), C.POINTER(gbm3d_opts),
                                      C.POINTER(gbm3d_opts), C.c_int]),
    "gbm3d_pilot_param_count": (C.c_int, []),
    "gbm3d_pilot_set_params": (C.c_int, [_P, _P]),
    "gbm3d_pilot_get_params": (C.c_int, [_P, _P]),
    "gbm3d_pilot_forward": (C.c_int, [_P, _P, _P, C.c_int, C.c_int, C.c_int, _P]),
    "gbm3d_pilot_train_step": (C.c_int, [_P, _P, _P, _P, C.c_int, C.c_int, C.c_int, C.c_float, _P]),
    "gbm3d_pilot_gradients": (C.c_int, [_P, _P, _P, _P, C.c_int, C.c_int, C.c_int, _P, _P]),
    "gbm3d_denoise_colored": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_double, _P, _P, C.POINTER(gbm3d_opts), _P,
                                        _P]),
    "gbm3d_matchBlocks_noalloc": (C.c_int, [_P, C.c_int, C.c_int, C.c_double, C.POINTER(gbm3d_opts), _P, _P, _P]),
}

_lib = None


def header_symbols() -> list[str]:
    """Function names declared in include/gbm3d.h."""
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(gbm3d_\w+)\s*\(", txt)))


def lib() -> C.CDLL:
    """Load libgbm3d.so (no fallback: raises if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing; build it with `python -m gbm3d_b200.build` "
                "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class Context:
    """A gbm3d_ctx bound to one CUDA device (one per host thread)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        rc = lib().gbm3d_ctx_create(device, C.byref(h))
        if rc != GBM3D_OK:
            raise GBM3DError(rc, f"cannot create a context on CUDA device {device}")
        self.h = h
        self.device = device

    def check(self, rc: int) -> None:
        if rc != GBM3D_OK:
            raise GBM3DError(rc, lib().gbm3d_last_error(self.h).decode())

    def close(self) -> None:
        if self.h:
            lib().gbm3d_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int | None) -> None:
        self.check(lib().gbm3d_ctx_set_stream(self.h, C.c_void_p(stream_ptr or 0)))

    def enable_timing(self, on: bool = True) -> None:
        self.check(lib().gbm3d_ctx_enable_timing(self.h, 1 if on else 0))

    def set_lanes(self, lanes: int = 1) -> None:
        """Streams the batched form's mixed submission runs on at once (1..16)."""
        self.check(lib().gbm3d_ctx_set_lanes(self.h, int(lanes)))

    def set_tc_wait(self, cycles: int = 0) -> None:
        """Limit (SM clocks) of each wait in the tensor-core matcher; 0 = about
        two seconds.  Negative: a probe of the give-up path (every CTA waits
        -cycles clocks on a barrier that nothing completes, then gives up)."""
        self.check(lib().gbm3d_ctx_set_tc_wait(self.h, int(cycles)))

    def tc_stats(self, enable: bool = True, read: bool = True) -> list[int] | None:
        """Candidates per reference left by the tensor-core matcher's bound:
        33 buckets of 8 (the last: 256 or more).  Returns the counts since the
        last read (and resets them) when ``read``."""
        buf = (C.c_int32 * 33)()
        self.check(lib().gbm3d_ctx_tc_stats(self.h, 1 if enable else 0, buf if read else None))
        return [int(x) for x in buf] if read else None

    def stage_times(self) -> list[float]:
        buf = (C.c_float * 8)()
        n = lib().gbm3d_stage_times(self.h, buf, 8)
        return [float(buf[i]) for i in range(max(n, 0))]

    def synchronize(self) -> None:
        """Wait for the context's work, including gbm3d_denoise_async copies;
        raises on a non-finite input among the asynchronous calls."""
        self.check(lib().gbm3d_ctx_synchronize(self.h))

    def launch_count(self) -> int:
        return int(lib().gbm3d_last_launch_count(self.h))

    def kernel_time(self, name: str) -> tuple[int, float]:
        """(launches, total ms) of one kernel family in the last timed call."""
        t = C.c_float(0.0)
        n = lib().gbm3d_kernel_time(self.h, name.encode(), C.byref(t))
        return int(n), float(t.value)


_ctx: dict[int, Context] = {}


def context(device: int = 0) -> Context:
    if device not in _ctx:
        _ctx[device] = Context(device)
    return _ctx[device]
