"""The C-ABI library loads and exports every symbol include/*.h declares,
and the host-side argument checks follow the reference.  No kernel runs here."""
import ctypes
import glob
import os
import re

import pytest

from conftest import HAVE_GPU, ROOT

import algofft
from algofft import _lib


def _declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"GFFT_API\s+[\w\s\*]+?\b(gfft_\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = _declared_symbols()
    assert "gfft_plan_new" in names and "gfft_forward_batch" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in _declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_every_symbol():
    declared = set(_declared_symbols())
    bound = set(_lib.SIGNATURES)
    assert declared == bound, (declared - bound, bound - declared)


def test_status_strings_match_reference_sentinels():
    L = algofft.lib()
    # errors.go:6-30 messages
    assert L.gfft_status_string(1) == b"algo-fft: invalid FFT length"
    assert L.gfft_status_string(2) == b"algo-fft: nil slice"
    assert L.gfft_status_string(3) == b"algo-fft: slice length mismatch"
    assert L.gfft_status_string(4) == b"algo-fft: invalid stride"
    assert L.gfft_status_string(5) == b"algo-fft: invalid spectrum"
    assert L.gfft_status_string(6) == b"algo-fft: not implemented"


def test_exception_classes_map_status():
    for status, cls in [(1, algofft.ErrInvalidLength), (2, algofft.ErrNilSlice), (3, algofft.ErrLengthMismatch),
                        (4, algofft.ErrInvalidStride), (5, algofft.ErrInvalidSpectrum),
                        (6, algofft.ErrNotImplemented)]:
        with pytest.raises(cls):
            algofft.check(status)


def test_invalid_length_rejected_before_device():
    # n < 1 is ErrInvalidLength (plan.go:808-810) with or without a GPU.
    with pytest.raises(algofft.ErrInvalidLength):
        algofft.NewPlan(0)


@pytest.mark.skipif(HAVE_GPU, reason="checks the no-device path")
def test_no_device_reported_without_gpu():
    assert algofft.device_count() == 0
    with pytest.raises(algofft.ErrNoDevice):
        algofft.NewPlan(1024)
