"""Wisdom and autotuning: wisdom.go:13-82 and the measuring planner
(internal/fft/measure.go) over the C ABI."""
from __future__ import annotations

import ctypes
import json

from ._lib import check, lib


def _read_string(fn, *args) -> str:
    need = ctypes.c_size_t(0)
    check(fn(*args, None, 0, ctypes.byref(need)))
    buf = ctypes.create_string_buffer(max(1, need.value))
    check(fn(*args, buf, need.value, ctypes.byref(need)))
    return buf.value.decode()


def ImportWisdomFromString(data: str) -> None:
    """wisdom.go:63 ImportWisdomFromString."""
    check(lib().gfft_wisdom_import_string(data.encode()))


def ImportWisdom(filename: str) -> None:
    """wisdom.go:13 ImportWisdom."""
    check(lib().gfft_wisdom_import_file(filename.encode()))


def ExportWisdom(filename: str) -> None:
    """wisdom.go:30 ExportWisdom."""
    check(lib().gfft_wisdom_export_file(filename.encode()))


def ExportWisdomToString() -> str:
    return _read_string(lib().gfft_wisdom_export_string)


def ClearWisdom() -> None:
    """wisdom.go:72 ClearWisdom."""
    lib().gfft_wisdom_clear()


def WisdomLen() -> int:
    """wisdom.go:77 WisdomLen."""
    return int(lib().gfft_wisdom_len())


def Variants(n: int, precision: int = 0) -> list[str]:
    """Tokens of every compiled kernel variant for (precision, n)."""
    return [t for t in _read_string(lib().gfft_plan_variants, precision, n).split("\n") if t]


def Autotune(n: int, precision: int = 0, count: int = 0, iters: int = 10) -> dict:
    """Times every variant on the device, records the fastest as wisdom and
    returns {"variants": {token: median ms}, "best": token, ...}."""
    cap = 1 << 16  # one call: a second call would re-run the measurement
    buf = ctypes.create_string_buffer(cap)
    need = ctypes.c_size_t(0)
    check(lib().gfft_autotune(precision, n, count, iters, buf, cap, ctypes.byref(need)))
    return json.loads(buf.value.decode())
