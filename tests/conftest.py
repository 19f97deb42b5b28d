"""Shared fixtures.  Tests marked `gpu` need a CUDA device; everything else runs on CPU.

The product library (kerrtrace_b200/libkerrtrace.so) and the checker libraries
(oracle/libkt_oracle.so, oracle/_ref/*.so) are built by `python __graft_entry__.py` /
`__graft_entry__.build()`; where nvcc is present and they are missing they are built here.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running")


def _ensure_built():
    from kerrtrace_b200 import build as kbuild
    import oracle.build as obuild
    if not kbuild.LIB.exists():
        kbuild.build()
    if not obuild.ORACLE_LIB.exists():
        obuild.build_oracle()


_ensure_built()


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    return torch


@pytest.fixture(scope="session")
def kt():
    import kerrtrace_b200
    return kerrtrace_b200


@pytest.fixture(scope="session")
def orc():
    import oracle
    return oracle


def pytest_collection_modifyitems(config, items):
    # keep the file order stable: alphabetical by file, declaration order inside a file
    items.sort(key=lambda it: (str(it.fspath), 0))


os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
