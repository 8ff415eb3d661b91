"""Index arithmetic of the dense sym4 x Haar wavelet kernels and the patch-32
video matcher, replayed on the CPU for every size the launchers accept in a
sweep: one wrap of each periodic index is enough (the kernels wrap once
instead of taking a modulo), and every shared-memory and global index stays
inside its buffer.  The formulas are those of k_wav_analysis_dense<7, 16>,
k_wav_synthesis_dense<7> (gbm3d_b200/csrc/wavelet.cu, with the launchers'
size checks) and k_match_video<32> (gbm3d_b200/csrc/video.cu)."""
import itertools

R, T_AN, TP = 7, 16, 32  # filter reach, analysis tile (coefficients), synthesis tile (samples)


def analysis_ok(Ly, Lx, Lz, shift):
    """The launcher's condition for the dense analysis kernel."""
    return shift >= 0 and Ly >= 2 * T_AN + 7 + shift and Lx >= 2 * T_AN + 7 + shift and Lz >= 2 and shift + 1 <= Lz


def synthesis_ok(Oy, Ox, Oz, shift):
    return Oy >= 2 * TP + 8 and Ox >= 2 * TP + 8 and Oz >= 2 and 0 <= shift < min(Oy, Ox, Oz)


def once(v, L):
    assert -L <= v < 2 * L, (v, L)  # a single wrap brings v into [0, L)
    return v + L if v < 0 else (v - L if v >= L else v)


def check_analysis(Ly, Lx, Lz, shift):
    NY = 2 * T_AN + R
    Oy, Ox, Oz = Ly // 2, Lx // 2, Lz // 2
    for qy0 in range(0, Oy, T_AN):
        y0 = 2 * qy0 - R - shift
        for yy in (0, NY - 1):  # the extremes of the staged rows
            assert 0 <= once(y0 + yy, Ly) < Ly
    for qx0 in range(0, Ox, T_AN):
        x0 = 2 * qx0 - R - shift
        for xx in (0, NY - 1):
            assert 0 <= once(x0 + xx, Lx) < Lx
    for qz in range(Oz):
        assert 0 <= once(2 * qz - shift, Lz) < Lz and 0 <= once(2 * qz - 1 - shift, Lz) < Lz
    # x-pass reads tz[fz][2 qx + R - u][yy], y-pass tx[comb][qx][2 qy + R - u]
    for qx, u in itertools.product((0, T_AN - 1), (0, R)):
        assert 0 <= 2 * qx + R - u < NY
    for qy, u in itertools.product((0, T_AN - 1), (0, R)):
        assert 0 <= 2 * qy + R - u < NY


def check_synthesis(Oy, Ox, Oz, shift):
    NQ = (TP - 1 + R) // 2 + 1
    Iy, Ix = Oy // 2, Ox // 2
    for py0 in range(0, Oy, TP):
        for qyl in (0, NQ - 1):
            assert 0 <= once(py0 // 2 + qyl, Iy) < Iy
        for py in (0, min(TP, Oy - py0) - 1):  # outputs past the size are skipped
            assert 0 <= once(py0 + py - shift, Oy) < Oy
    for px0 in range(0, Ox, TP):
        for qxl in (0, NQ - 1):
            assert 0 <= once(px0 // 2 + qxl, Ix) < Ix
    for qz in range(Oz // 2):
        for which in (0, 1):
            pz = once(2 * qz - which, Oz)
            assert 0 <= once(pz - shift, Oz) < Oz
    # y-pass: B[.][qxl][j + (u + 1) / 2] for j < TP / 2; x-pass: Y[.][(px + u) / 2][py]
    assert TP // 2 - 1 + (R + 1) // 2 < NQ
    assert (TP - 1 + R) // 2 < NQ


def test_dense_wavelet_indices_single_wrap():
    n = 0
    for Ly, Lx in itertools.product((40, 46, 48, 64, 72, 96, 184, 368, 736, 1280, 1024), repeat=2):
        for Lz, shift in ((2, 0), (4, 1), (8, 0), (16, 1), (16, 3)):
            if analysis_ok(Ly, Lx, Lz, shift):
                check_analysis(Ly, Lx, Lz, shift)
                n += 1
            if synthesis_ok(Ly, Lx, Lz, shift):
                check_synthesis(Ly, Lx, Lz, shift)
                n += 1
    assert n > 200


def test_video_matcher_patch32_window_indices():
    """k_match_video<32>: lane a = candidate row, warp w the 8 columns from
    b0 = 8 w; the sliding row reads window columns b0 .. b0 + 38 of rows
    a + r, inside the 64 x 64 window; the keys of its 8 candidates are
    distinct and cover the frame's 1024."""
    D, WD, NB = 32, 64, 8
    keys = set()
    for tid in range(128):
        a, b0 = tid & 31, (tid >> 5) * NB
        assert a + D - 1 < WD  # rows a + r
        assert b0 + (D - 1) + NB - 1 < WD  # the last column the row slides to
        keys.update(a + (b0 + q) * D for q in range(NB))
    assert keys == set(range(D * D))
