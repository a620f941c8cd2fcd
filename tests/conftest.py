"""Test configuration.

* registers the ``gpu`` marker (tests that need a B200);
* loads oracle/librecord_xerbla.so with RTLD_GLOBAL before anything else, so the
  xerbla_ calls of both Eigen's reference BLAS and libeigen_b200.so resolve to the
  recorder and argument-error info codes can be checked (blas/xerbla.cpp:18-20 is
  weak; so is the product's).
"""
from __future__ import annotations

import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
TESTS = Path(__file__).resolve().parent
if str(TESTS) not in sys.path:
    sys.path.insert(0, str(TESTS))

import _helpers  # noqa: E402

_helpers.load_xerbla_recorder()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")
