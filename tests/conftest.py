"""Shared pytest setup.

Markers: ``gpu`` -- needs a CUDA device (a B200 for the parity and timing
tests).  Everything else runs on a CPU-only host.
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run on a B200)")
