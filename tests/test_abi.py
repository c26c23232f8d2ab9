"""The C-ABI library loads and exports every symbol include/sunset_gpu.h declares (no GPU
calls), and the host-side mirror fails loudly when no GPU is present."""
import ctypes
import os
import re

import pytest

from sunset_viscoelastic_b200 import labfm

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "sunset_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sunset_[A-Za-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = labfm.load_library()
    names = declared_symbols()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(labfm.ABI_SYMBOLS)


def test_library_is_built_for_sm100a():
    # the build compiles every source for sm_100a SASS only (no PTX for other targets)
    from sunset_viscoelastic_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


@pytest.mark.gpu
def test_kernels_run_as_sm100_binaries():
    # what the CUDA runtime reports for a kernel of the loaded library
    lib = labfm.load_library()
    assert lib.sunset_kernel_binary_version(0) == 100


def test_version_and_error_paths_without_gpu():
    lib = labfm.load_library()
    assert lib.sunset_version() == 1
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(labfm.SunsetError):
        labfm.Sunset()


def test_bad_configuration_is_rejected_before_device_work():
    lib = labfm.load_library()
    cfg = labfm.SunsetConfig()
    cfg.form, cfg.morder, cfg.forder, cfg.Re, cfg.Wi, cfg.Ma = 0, 5, 5, 1.0, 1.0, 0.1
    h = ctypes.c_void_p()
    rc = lib.sunset_create(ctypes.byref(cfg), ctypes.byref(h))
    assert rc == -4 and b"orders" in lib.sunset_last_error(h)
    lib.sunset_destroy(h)
