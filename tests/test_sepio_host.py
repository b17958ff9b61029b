"""The reference's on-disk format (binWrite / binRead, src/include/IO.hpp:
179-429) through fwi2d_b200.sepio.

tests/golden/sep/model_ref.H (+ model_ref.H@) was written by the reference's
own binWrite (tests/golden/make_golden.py:sep_case).  The library must read it
back exactly, write the same header text and binary for the same cube, and,
where the reference build is present, the reference must read the library's
files.
"""
import os
import sys

import numpy as np
import pytest

import oracle as O
from fwi2d_b200 import sepio

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLD)
import make_golden as G  # noqa: E402


def test_read_reference_file():
    a, axes = sepio.read_bin(os.path.join(GOLD, "sep", "model_ref.H"))
    assert np.array_equal(a, G.sep_values())
    assert [(n, o, d) for n, o, d, _ in axes] == [(16, 0.0, 0.005), (20, 0.5, 0.005), (3, 0.0, 1.0)]


def test_write_matches_reference_bytes(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    sepio.write_bin(G.sep_values(), "model_ref.H", G.SEP_AXES, datapath=".")
    for name in ("model_ref.H", "model_ref.H@"):
        with open(os.path.join(GOLD, "sep", name), "rb") as f, open(name, "rb") as g:
            assert f.read() == g.read(), name


def test_trailing_unit_axes_and_size_check(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    x = np.arange(12, dtype=np.float32).reshape(1, 3, 4)
    sepio.write_bin(x, "t.H", datapath=".")
    a, axes = sepio.read_bin("t.H")
    assert a.shape == (3, 4) and len(axes) == 2           # n3 = 1 dropped, as binRead does
    a3, axes3 = sepio.read_bin("t.H", ndim0=3)
    assert a3.shape == (1, 3, 4) and len(axes3) == 3
    with open("t.H@", "ab") as f:
        f.write(b"\0\0\0\0")
    with pytest.raises(ValueError):
        sepio.read_bin("t.H")


@pytest.mark.skipif(not O.have_reference(32), reason="oracle/_ref is not built")
def test_reference_reads_library_file(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    x = np.random.default_rng(9).standard_normal((2, 7, 5)).astype(np.float32)
    sepio.write_bin(x, "lib.H", [(0.1, 0.01), (2.0, 0.02), (0.0, 1.0)], datapath=str(tmp_path))
    a, axes = O.Reference(32).bin_read("lib.H")
    assert np.array_equal(a, x)
    assert [n for n, _, _ in axes] == [5, 7, 2]
    assert np.allclose([o for _, o, _ in axes], [0.1, 2.0, 0.0]) and np.allclose([d for _, _, d in axes], [0.01, 0.02, 1])
