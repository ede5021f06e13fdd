"""The mcstar-libs-named C++ headers (include/mcstar/) are a drop-in for the reference's
source-level API on the stepper path: a host program written against cuda/, cuda/kernels/
and common/ compiles unchanged, in FP32 and FP64, and links libpfc_b200 alone."""
import os
import shutil

import pytest

from conftest import ROOT, build_shim_driver

HEADERS = [
    "cuda/array_abstraction.hpp", "cuda/cufft_wrapper.hpp", "cuda/noise.hpp", "cuda/cutiming.hpp",
    "cuda/potentials.hpp", "cuda/kernels/common.hpp", "cuda/kernels/eom.hpp", "cuda/kernels/psi3_split.hpp",
    "cuda/kernels/norm.hpp", "cuda/kernels/findpeaks.hpp", "cuda/kernels/findpeaks_2d.hpp",
    "cuda/kernels/eom-exp.hpp", "cuda/kernels/el.hpp", "cuda/kernels/el-exp.hpp", "common/pfc.hpp",
    "common/maximum_struct.hpp", "common/technicalities.hpp", "common/cu_error.hpp",
    "bond-order-analysis/bond-order.hpp",
]


def test_reference_named_headers_present():
    for h in HEADERS:
        assert os.path.isfile(os.path.join(ROOT, "include", "mcstar", h)), h


def _lib_built():
    return os.path.exists(os.path.join(ROOT, "mcstar-libs_b200", "mcstar_b200", "lib", "libpfc_b200.so"))


@pytest.mark.skipif(shutil.which("nvcc") is None and not os.path.exists("/usr/local/cuda/bin/nvcc"),
                    reason="nvcc not available")
@pytest.mark.parametrize("flt", ["float", "double"])
@pytest.mark.parametrize("driver", ["driver_step.cu", "driver_relax.cu", "driver_lowpass.cu"])
def test_reference_style_driver_compiles_and_links(flt, driver, tmp_path):
    if not _lib_built():
        pytest.skip("libpfc_b200.so not built")
    rc, out = build_shim_driver(flt, tmp_path / f"drv_{flt}", os.path.join(ROOT, "tests", "shim", driver))
    assert rc == 0, out[-3000:]
    assert "warning" not in out.lower(), out[-3000:]
