import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "oracle"), os.path.join(ROOT, "sbd-ykt_b200"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)
# the oracle module must win over the oracle/ directory name
sys.path.remove(os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
