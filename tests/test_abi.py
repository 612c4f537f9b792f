"""The C ABI library: built for sm_100a, loadable without a GPU, exporting every
symbol include/linqt_gpu.h declares, and reporting errors instead of aborting."""
import ctypes
import os
import re

import numpy as np
import pytest

import linqt_b200 as lq
from linqt_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "linqt_gpu.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(linqt_[a-z0-9_]+)\s*\(", hdr)))


def test_library_built_and_loads():
    assert os.path.exists(_lib.LIB_PATH)
    L = _lib.load()
    assert L.linqt_abi_version() == _lib.ABI_VERSION == 3


def test_every_declared_symbol_is_exported():
    L = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing
    # and the ctypes table covers the whole header
    assert set(names) == set(_lib.SIGNATURES)


def test_library_targets_sm100a():
    # nvcc records the target in the fatbin section name of the ELF; the build flags say it too
    from linqt_b200 import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)


def test_host_only_entry_points_match_oracle(oracle_lib):
    rng = np.random.default_rng(0)
    mu = rng.normal(size=64) + 1j * rng.normal(size=64)
    got = lq.jackson1d(mu, 8.0, 150.0)
    want = oracle_lib.jackson1d(mu, 8.0, 150.0)
    assert len(got) == len(want)
    assert np.abs(got - want).max() < 1e-15
    mu2 = rng.normal(size=(50, 40)) + 1j * rng.normal(size=(50, 40))
    got2 = lq.jackson2d(mu2, 4.9, 50.0, 80.0)
    want2 = oracle_lib.jackson2d(mu2, 4.9, 50.0, 80.0)
    assert got2.shape == want2.shape
    assert np.abs(got2 - want2).max() < 1e-15


def test_errors_without_gpu_are_codes_not_aborts():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(lq.LinqtError) as e:
        lq.Session(0)
    assert e.value.code in (-1, -2)
    with pytest.raises(lq.LinqtError) as e:
        lq.jackson1d(np.ones(4), 8.0, -1.0)
    assert e.value.code == -1
