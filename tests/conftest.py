"""Test configuration: the ``gpu`` marker and import paths.

The product package lives in ``blind-spiking-lstm_b200/`` (a source root
holding the ``tfhe_b200`` Python package and its CUDA sources); the oracle in
``oracle/`` is the checker.
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_ROOT = os.path.join(ROOT, "blind-spiking-lstm_b200")
for p in (ROOT, PKG_ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
