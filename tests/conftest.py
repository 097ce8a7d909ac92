import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


# The reference's param.in, where the reference tree sits beside this checkout's build
# machine; tests that read it are skipped otherwise.
_PARAM_IN = os.path.join(os.path.dirname(ROOT), "reference", "source", "param.in")
if "GAZPART_REFERENCE_PARAM_IN" not in os.environ and os.path.exists(_PARAM_IN):
    os.environ["GAZPART_REFERENCE_PARAM_IN"] = _PARAM_IN


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
