"""fg_probe_peak: the measured dense rate of each compute pipe, the
denominator of the bench's roofline fractions."""
import pytest


@pytest.mark.gpu
def test_probe_peaks_are_plausible(fg):
    """fg_probe_peak: each pipe's measured dense rate lies between a quarter
    of and a little above the B200 spec-sheet figure (INT8 4.5 POPS, BF16
    2.25 PFLOP/s, FP64 40 TFLOP/s, FP32 FFMA 74 TFLOP/s), and the context
    stays usable (no bounded wait ran out)."""
    import ctypes as C
    from ferray_b200 import _lib as L
    ctx = fg.default_context()
    for which, spec in ((L.FG_PROBE_INT8, 4.5e15), (L.FG_PROBE_BF16, 2.25e15),
                        (L.FG_PROBE_FP64, 40e12), (L.FG_PROBE_FFMA, 74e12)):
        v = C.c_double()
        assert ctx._lib.fg_probe_peak(ctx.handle, which, C.byref(v)) == 0, ctx._lib.fg_last_error()
        assert spec / 4 < v.value < spec * 1.3, (which, v.value)
    assert ctx._lib.fg_probe_peak(ctx.handle, 99, C.byref(v)) == L.FG_ERR_INVALID
