"""pytest configuration: the ``gpu`` marker and import paths.

``-m "not gpu"`` runs the oracle-vs-golden checks, host logic and the
C-ABI symbol checks (no device needed); ``-m gpu`` runs the parity tests
proper, which call libfk through its C ABI on a CUDA device and fail
loudly if the library or the device is missing.
"""

import pathlib
import sys

ROOT = pathlib.Path(__file__).resolve().parents[1]
PKG = ROOT / "first-knowns_b200"
for p in (str(ROOT), str(PKG), str(ROOT / "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs a CUDA device (B200) and libfk.so")
    config.addinivalue_line(
        "markers", "slow: long-running parity sweep")
