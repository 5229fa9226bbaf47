"""The fused path's in-place transform stages (decimation in frequency forward, in time
inverse, digit-reversed spectra in between), built for the host from the same header, against
numpy's circular convolution at every length kind the path serves."""
import ctypes as ct
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("fz") / "libfz_host.so")
    nvcc = os.environ.get("TACO_NVCC", "/usr/local/cuda/bin/nvcc")
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    subprocess.run([nvcc, "-std=c++17", "-O2", "-shared", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                    "-I", os.path.join(ROOT, "taco_b200", "csrc"), "-x", "cu",
                    os.path.join(HERE, "native", "fz_host_harness.cu"), "-o", out], check=True)
    lib = ct.CDLL(out)
    lib.fz_host_convolve.argtypes = [ct.c_int, ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p]
    return lib


@pytest.mark.parametrize("N", [8, 12, 40, 96, 160, 1280, 2048, 2560, 3072, 10240, 16384, 20480, 24576])
def test_fused_stages_convolve_like_numpy(harness, N):
    rng = np.random.default_rng(N)
    a = rng.normal(size=N) + 1j * rng.normal(size=N)
    b = rng.normal(size=N) + 1j * rng.normal(size=N)
    ref = np.fft.ifft(np.fft.fft(a) * np.fft.fft(b))
    for fp32, radix, tol in ((1, 16, 1e-6), (1, 8, 1e-6), (0, 8, 1e-13)):  # FP64 plans stop at radix 8
        out = np.empty(N, np.complex128)
        rc = harness.fz_host_convolve(N, fp32, radix, a.ctypes.data, b.ctypes.data, out.ctypes.data)
        assert rc == 0
        err = np.linalg.norm(out - ref) / np.linalg.norm(ref)
        assert err <= tol, (N, fp32, radix, err)
