import pathlib
import sys

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    # The C restatement is part of the checker; build it on demand.
    import oracle
    if not oracle.PORT_SO.exists():
        oracle.build(reference=False)
    from neospice_b200 import build as nb
    if not nb.LIB.exists():
        nb.build()
