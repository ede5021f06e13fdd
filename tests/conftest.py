import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "mcstar-libs_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libpfc_b200.so")


def pytest_collection_modifyitems(config, items):
    import torch
    if torch.cuda.is_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


SHIM_DRIVER = os.path.join(ROOT, "tests", "shim", "driver_step.cu")
LIB_DIR = os.path.join(ROOT, "mcstar-libs_b200", "mcstar_b200", "lib")


def build_shim_driver(flt, out, source=SHIM_DRIVER):
    """Compiles a driver of tests/shim/ (default driver_step.cu) against the
    mcstar-libs-named headers (include/mcstar) and libpfc_b200 with FLOAT=flt;
    returns (returncode, output)."""
    import shutil
    import subprocess
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cmd = [nvcc, "-std=c++17", "-O2", f"-DFLOAT={flt}", "-gencode", "arch=compute_100a,code=sm_100a",
           "-Xcompiler", "-Wall", "-I", os.path.join(ROOT, "include", "mcstar"), "-I", os.path.join(ROOT, "include"),
           source, "-L", LIB_DIR, "-lpfc_b200", f"-Xlinker", f"-rpath={LIB_DIR}", "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    return r.returncode, r.stdout + r.stderr


def ref_lib(dtype):
    """The reference's own cuFFT path (oracle/_ref), or None when it was not built."""
    import ctypes
    import numpy as np
    name = "libref_pfc_f32.so" if np.dtype(dtype) == np.float32 else "libref_pfc_f64.so"
    path = os.path.join(REF_DIR, name)
    if not os.path.exists(path):
        return None
    L = ctypes.CDLL(path)
    pre = "ref32_" if np.dtype(dtype) == np.float32 else "ref64_"
    P, D, I = ctypes.c_void_p, ctypes.c_double, ctypes.c_int
    sig = {
        "create": ([I, I, I, ctypes.c_ulonglong], P), "destroy": ([P], None),
        "set_kpsi": ([P, P], None), "get_kpsi": ([P, P], None), "r2c": ([P, P, P], None),
        "c2r": ([P, P, P], None), "step": ([P, I, D, D, D, D, D, D, D, I], None),
        "time_steps": ([P, I, D, D, D, D, D, D, D, I], ctypes.c_float), "get_psi": ([P, P], None),
        "free_energy": ([P, D, D, D, D, D, D, D, P], ctypes.c_float),
        "findpeaks": ([P, D, D, D, D, D, D, D, D, ctypes.c_char_p, ctypes.c_char_p], None),
        "noise_kspace": ([P, P], None),
    }
    fns = {}
    for k, (a, r) in sig.items():
        f = getattr(L, pre + k)
        f.argtypes = a
        f.restype = r
        fns[k] = f
    return fns
