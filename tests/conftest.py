import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "mujoco-mlx-cpp_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs through the C ABI on the CUDA engine)")


@pytest.fixture(scope="session")
def quad_xml():
    import mjb200
    return mjb200.models.quadruped_xml()


@pytest.fixture(scope="session")
def quad_model(quad_xml):
    import mjb200
    return mjb200.load_model_from_string(quad_xml)
