"""Test configuration: import paths and the `gpu` marker.

`-m "not gpu"` runs the oracle pins, host logic and C-ABI load checks on CPU;
`-m gpu` runs the parity tests on a B200 through the C-ABI.
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "cuda-dolfinx_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (sm_100a)")


_built = []


def ensure_library():
    """(Re)build the shared library when sources are newer (incremental; nvcc
    cross-compiles on CPU-only hosts).  Where no nvcc exists the prebuilt
    library is used as is."""
    lib = os.path.join(PKG, "lib", "libcudolfinx_b200.so")
    if not _built:
        import shutil

        if shutil.which("nvcc") or os.path.exists("/usr/local/cuda/bin/nvcc") or not os.path.exists(lib):
            import build  # cuda-dolfinx_b200/build.py

            build.build()
        _built.append(True)
    return lib
