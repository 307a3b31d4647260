import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

ORACLE_LIB = os.path.join(ROOT, "oracle", "liboracle_tc.so")
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
REF_LIB = os.path.join(REF_DIR, "libtopos_codec_ref.so")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def _reference_dir():
    """The reference checkout (CPU tests only): TOPOS_REFERENCE_DIR, else the
    directory the oracle recipe built oracle/_ref from; None when neither."""
    env = os.environ.get("TOPOS_REFERENCE_DIR")
    if env:
        return env
    rec = os.path.join(REF_DIR, "SOURCE_DIR")
    if os.path.exists(rec):
        with open(rec) as f:
            d = f.read().strip()
        return d or None
    return None


REFERENCE_DIR = _reference_dir()


def reference_path(*parts):
    """A file of the reference checkout, or a path that does not exist."""
    return os.path.join(REFERENCE_DIR, *parts) if REFERENCE_DIR else os.path.join(REF_DIR, "missing", *parts)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C-ABI")


def _gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def built():
    """Builds the product library and the oracle (idempotent)."""
    from topos_codec_b200 import _build
    _build.build_library()
    if not os.path.exists(ORACLE_LIB):
        _build.build_oracle()
    return True


@pytest.fixture(scope="session")
def product(built):
    from topos_codec_b200 import binding as B
    return B.ToposCodec(B.PRODUCT_LIBRARY)


@pytest.fixture(scope="session")
def oracle(built):
    from topos_codec_b200 import binding as B
    return B.ToposCodec(ORACLE_LIB)


@pytest.fixture(scope="session")
def reference():
    from topos_codec_b200 import binding as B
    if not os.path.exists(REF_LIB):
        pytest.skip("reference library not built (oracle/_ref)")
    return B.ToposCodec(REF_LIB)
