import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
if str(ROOT / "tests") not in sys.path:
    sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Builds libmvbt.so, the workload generator and the oracle if they are missing or stale (nvcc cross-compiles here)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("mvbt_build", ROOT / "mvgpubtree_b200" / "build.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.build()
    from workload.build import build as build_workload
    build_workload()
    from oracle.build import build as build_oracle
    build_oracle()
    spec = importlib.util.spec_from_file_location("cpp_build", ROOT / "tests" / "cpp" / "build.py")
    cpp = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(cpp)
    cpp.build_user_kernels()
    yield
