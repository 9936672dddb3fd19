"""pytest configuration: the ``gpu`` marker and import paths.

GPU tests need a CUDA device and the built ``libfhs_b200.so``; everything
else runs on CPU.
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "faceted-hypersara_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built libfhs_b200.so")
