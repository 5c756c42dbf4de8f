"""Wisdom text format and store semantics (internal/planner/wisdom.go:96-205),
host-only: no kernel runs here."""
import os

import pytest

import algofft


@pytest.fixture(autouse=True)
def _clean():
    algofft.ClearWisdom()
    yield
    algofft.ClearWisdom()


def test_roundtrip_and_sorting():
    text = ("# comment\n\n"
            "4096:0:100:gpu-sm100-p2-n4096-e16:1700000000\n"
            "1024:1:100:gpu-sm100-p2-n1024-e16:1700000001\n"
            "1024:0:100:gpu-sm100-p2-n1024-e32:1700000002\n")
    algofft.ImportWisdomFromString(text)
    assert algofft.WisdomLen() == 3
    out = algofft.ExportWisdomToString().splitlines()
    # sorted by size, then precision, then features (wisdom.go:103-113)
    assert out == ["1024:0:100:gpu-sm100-p2-n1024-e32:1700000002",
                   "1024:1:100:gpu-sm100-p2-n1024-e16:1700000001",
                   "4096:0:100:gpu-sm100-p2-n4096-e16:1700000000"]


def test_same_key_overwrites():
    algofft.ImportWisdomFromString("64:0:100:a:1\n64:0:100:b:2\n")
    assert algofft.WisdomLen() == 1
    assert algofft.ExportWisdomToString().strip() == "64:0:100:b:2"


@pytest.mark.parametrize("bad", ["1024:0:100:x\n", "1024:0:100:x:1:2\n", "abc:0:100:x:1\n",
                                 "1024:0:100:x:ts\n", "1024:999:100:x:1\n"])
def test_malformed_lines_rejected_atomically(bad):
    algofft.ImportWisdomFromString("8:0:100:keep:1\n")
    with pytest.raises(algofft.ErrWisdom):
        algofft.ImportWisdomFromString("16:0:100:new:1\n" + bad)
    # a failed import changes nothing
    assert algofft.ExportWisdomToString().strip() == "8:0:100:keep:1"


def test_file_roundtrip(tmp_path):
    algofft.ImportWisdomFromString("2048:0:100:gpu-sm100-p2-n2048-e16:5\n")
    p = str(tmp_path / "w.txt")
    algofft.ExportWisdom(p)
    algofft.ClearWisdom()
    assert algofft.WisdomLen() == 0
    algofft.ImportWisdom(p)
    assert algofft.WisdomLen() == 1
    with pytest.raises(algofft.ErrWisdom):
        algofft.ImportWisdom(str(tmp_path / "missing.txt"))


def test_variants_listed_without_device():
    v = algofft.Variants(1024)
    assert "gpu-sm100-p2-n1024-e32" in v and "gpu-sm100-tp-32x32-t8192-e16" not in v
    v = algofft.Variants(1 << 20)
    assert any(t.startswith("gpu-sm100-tp-1024x1024-") for t in v)
    # 7-smooth lengths: runtime-radix schedules against Bluestein
    assert algofft.Variants(1000) == ["gpu-sm100-mixed-n1000", "gpu-sm100-mixr-n1000", "gpu-sm100-mixed2-25x40",
                                      "gpu-sm100-bluestein-n1000"]
    assert algofft.Variants(1009) == []  # a prime: Bluestein is the only schedule
