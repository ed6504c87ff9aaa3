"""The library's measurement probes (roofline denominators and the FP64 /
INT8 overlap figure) run and return sane numbers."""

import ctypes

import pytest

pytestmark = pytest.mark.gpu


def test_peak_probes(negf):
    lib = negf.load()
    d1, d2, d3 = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    negf._lib.check(lib.negf_probe_fp64_peak(ctypes.byref(d1), ctypes.byref(d2)))
    negf._lib.check(lib.negf_probe_int8_peak(ctypes.byref(d3)))
    assert 1.0 < max(d1.value, d2.value) < 200.0      # TFLOP/s
    assert 100.0 < d3.value < 20000.0                 # TOP/s


def test_fp64_int8_overlap_probe(negf):
    lib = negf.load()
    a, b, m = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    negf._lib.check(lib.negf_probe_fp64_int8_overlap(ctypes.byref(a), ctypes.byref(b), ctypes.byref(m)))
    assert a.value > 0 and m.value > 0
    # FP64 work beside the MMA stream never finishes sooner than alone
    assert b.value >= 0.9 * a.value
