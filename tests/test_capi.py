"""The C ABI on a machine without a GPU: libmjb200.so loads, exports every
function the public headers declare, refuses what it does not implement with
a message, and fails cleanly (NULL + mjb200_last_error) where a device is
needed.  No compute call runs here."""
import ctypes as C
import os
import re

import pytest

import mjb200
from mjb200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include", "mjmlx")
DECL = re.compile(r"(?:MJB_API|MJMLX_API)\s+[^;(]*?\b(\w+)\s*\(", re.S)


def declared_functions():
    names = []
    for h in sorted(os.listdir(INCLUDE)):
        if h.endswith(".h"):
            with open(os.path.join(INCLUDE, h)) as f:
                src = re.sub(r"/\*.*?\*/", "", f.read(), flags=re.S)
            src = "\n".join(line for line in src.splitlines() if not line.lstrip().startswith("#"))
            names += [n for n in DECL.findall(src)]
    return names


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) > 80
    assert "mjb200_batched_step_noalloc" in names and "mjb_batched_step" in names and "mjmlx_batched_step_n" in names
    lib = C.CDLL(capi.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_backend_types():
    lib = capi.lib
    lib.mjb_create_backend.restype = C.c_void_p
    lib.mjb_create_backend.argtypes = [C.c_int]
    lib.mjb_free_backend.argtypes = [C.c_void_p]
    lib.mjb_backend_type.argtypes = [C.c_void_p]
    assert lib.mjb_create_backend(0) is None           # MJB_BACKEND_CPU: MuJoCo C is not in this library
    assert "MJB_BACKEND_CPU" in capi.last_error()
    for t in (1, 2):                                     # MJB_BACKEND_MLX (GPU engine), MJB_BACKEND_CUDA
        b = lib.mjb_create_backend(t)
        assert b
        assert lib.mjb_backend_type(b) == t
        lib.mjb_free_backend(b)
    assert lib.mjb_create_backend(7) is None


def test_cpu_only_create_is_refused(quad_model):
    with pytest.raises(RuntimeError) as e:
        _create_cpu(quad_model)
    assert "use_gpu = 0" in str(e.value)


def _create_cpu(model):
    cfg = capi.MjmlxBatchedConfig()
    cfg.num_envs, cfg.integrator, cfg.use_gpu, cfg.solver_iterations, cfg.domain_rand = 4, 0, 0, 0, 0
    fn = capi.lib.mjmlx_batched_create
    h = fn(model.handle, C.byref(cfg))
    if not h:
        raise RuntimeError(capi.last_error())
    return h


def test_create_without_a_gpu_fails_cleanly(quad_model):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(RuntimeError) as e:
        mjb200.BatchedSim(quad_model, 4)
    assert str(e.value)


def test_default_engine_config():
    c = capi.engine_config()
    assert c.lockstep == 1 and c.use_graph == 1 and c.warmstart >= 0
    assert c.tolerance <= 0  # <= 0 keeps the model's own solver tolerance
    assert c.ncon_max == 0 and c.nefc_max == 0 or (c.ncon_max > 0 and c.nefc_max > 0)


def test_model_info_and_null_handling(quad_model):
    info = capi.lib.mjmlx_model_info(quad_model.handle)
    assert (info.nq, info.nv, info.nu, info.nbody, info.ngeom) == (19, 18, 12, 14, 14)
    # NULL handles are rejected, not dereferenced
    null = capi.lib.mjmlx_model_info(None)
    assert (null.nq, null.nv) == (0, 0)
    assert capi.lib.mjmlx_name2id(None, 1, b"trunk") == -1


def test_camera_api_is_exported_and_refuses():
    """The reference's camera renderer is graphics (Vulkan); the entry points
    exist so its callers link, and they refuse with a message."""
    lib = C.CDLL(capi.LIB_PATH)
    lib.mjmlx_camera_create.restype = C.c_void_p
    lib.mjmlx_camera_create.argtypes = [C.c_void_p, C.c_int, C.c_int]
    assert lib.mjmlx_camera_create(None, 64, 48) is None
    assert "graphics" in capi.last_error()
    for fn in ("mjmlx_camera_render", "mjmlx_camera_gpu_copy"):
        getattr(lib, fn).argtypes = [C.c_void_p]
        assert getattr(lib, fn)(None) == -1
    lib.mjmlx_camera_count.argtypes = [C.c_void_p]
    lib.mjmlx_camera_gpu_supported.argtypes = [C.c_void_p]
    assert lib.mjmlx_camera_count(None) == 0 and lib.mjmlx_camera_gpu_supported(None) == 0
    lib.mjmlx_camera_free.argtypes = [C.c_void_p]
    lib.mjmlx_camera_free(None)
