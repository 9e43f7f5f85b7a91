import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds the oracle and the CUDA library once per session (no-op when fresh)."""
    import oracle
    from mjolnir_b200 import build
    if not os.path.exists(oracle.ORACLE_SO):
        oracle.build()
    build.build()
    yield


def golden_cases():
    """{name: (SystemDesc, fixture dict)} for every committed golden fixture;
    the description is rebuilt by the generating script and takes the stored
    coordinates."""
    import importlib.util
    import numpy as np
    path = os.path.join(ROOT, "tests", "golden", "make_golden.py")
    spec = importlib.util.spec_from_file_location("make_golden", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    out = {}
    for name, (d, _vv) in mod.cases().items():
        fx = dict(np.load(os.path.join(ROOT, "tests", "golden", name + ".npz")))
        d.pos = fx["pos"].copy()
        d.vel = fx["vel"].copy()
        out[name] = (d, fx)
    return out


def rel_rms(a, b):
    """sqrt(sum |a-b|^2 / sum |b|^2), the relative RMS error of a vs b."""
    import numpy as np
    den = float((np.asarray(b) ** 2).sum())
    num = float(((np.asarray(a) - np.asarray(b)) ** 2).sum())
    return (num / den) ** 0.5 if den > 0 else num ** 0.5


def sha256(a) -> str:
    import hashlib
    import numpy as np
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def config_cases():
    """{name: (SystemDesc, vv_dt, subset, fixture dict)} for the
    configuration-size fixtures of tests/golden/make_configs.py; each system is
    rebuilt by the same seeded builders, and its coordinates must hash to the
    stored SHA-256 (the fixtures do not store the inputs)."""
    import importlib.util
    import numpy as np
    path = os.path.join(ROOT, "tests", "golden", "make_configs.py")
    spec = importlib.util.spec_from_file_location("make_configs", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    out = {}
    for name, (d, dt, sub) in mod.cases().items():
        fx = dict(np.load(os.path.join(ROOT, "tests", "golden", name + ".npz")))
        assert sha256(d.pos) == str(fx["pos_sha"]) and sha256(d.vel) == str(fx["vel_sha"]), \
            f"{name}: the seeded builders no longer make the fixture's system"
        out[name] = (d, dt, sub, fx)
    return out
