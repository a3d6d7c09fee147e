"""The allocation-free GEMM entry point, checked against numpy and against the
regular entry point.

Some callers of this library cannot call cudaMalloc (their device memory is
owned by a host framework's pool, or they run where cudaMalloc/cudaFree are
not allowed).  ``ipeps_gemm_f64_noalloc`` serves them: it takes device
pointers and keeps its split-K partial sums in a fixed device array instead
of allocating.  This file is named to be collected last; it passes on its own
in a fresh process and after the other tests.

The test allocates its own device buffers (with torch) - only the entry point
under test must not allocate, which is checked through the device's free
memory around repeated calls.  Its output is compared with ``A @ B`` (numpy,
FP64) and with the regular allocating entry point (``ipeps_tcon``, host
buffers) within the FP64 bar of the other contraction tests (1e-12 relative),
on two calls in a row.
"""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

IPEPS_OK, IPEPS_EINVAL = 0, 4


def _noalloc(lib):
    f = lib.ipeps_gemm_f64_noalloc
    f.argtypes = [ct.c_char, ct.c_char, ct.c_int64, ct.c_int64, ct.c_int64, ct.c_double, ct.c_void_p, ct.c_int64,
                  ct.c_void_p, ct.c_int64, ct.c_double, ct.c_void_p, ct.c_int64, ct.c_void_p]
    f.restype = ct.c_int
    return f


def _device_colmajor(torch, X):
    """Column-major copy of the numpy matrix X on the device (row-major X^T)."""
    return torch.tensor(np.ascontiguousarray(X.T), dtype=torch.float64, device="cuda")


def _torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_noalloc_gemm_matches_numpy_and_regular_entry_point(pkg):
    torch = _torch_cuda()
    lib = ct.CDLL(pkg.LIB_PATH)
    gemm = _noalloc(lib)
    rng = np.random.default_rng(2024)
    # skinny outputs with long K take the split-K path and hence the static
    # scratch; the 700 x 500 output (> 262144 elements) runs unsplit
    cases = [("N", "N", 120, 150, 6000), ("T", "N", 96, 200, 4096), ("N", "T", 700, 500, 3000)]
    inputs = []
    for opA, opB, m, n, k in cases:
        A = rng.standard_normal((m, k) if opA == "N" else (k, m))
        B = rng.standard_normal((k, n) if opB == "N" else (n, k))
        dA, dB = _device_colmajor(torch, A), _device_colmajor(torch, B)
        dC = torch.full((n, m), 7.0, dtype=torch.float64, device="cuda")  # beta = 0 must ignore this
        inputs.append((opA, opB, m, n, k, A, B, dA, dB, dC))
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    free = []
    for call in range(2):  # two calls in a row share (and reuse) the scratch
        for opA, opB, m, n, k, A, B, dA, dB, dC in inputs:
            st = gemm(opA.encode(), opB.encode(), m, n, k, 1.0, dA.data_ptr(), A.shape[0], dB.data_ptr(),
                      B.shape[0], 0.0, dC.data_ptr(), m, ct.c_void_p(stream))
            assert st == IPEPS_OK
            torch.cuda.synchronize()
            got = dC.cpu().numpy().T
            ref = (A if opA == "N" else A.T) @ (B if opB == "N" else B.T)
            assert np.allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max()), (call, opA, opB, m, n, k)
            if call == 1:
                # the regular entry point: tcon over the summed label, host buffers
                reg = pkg.tcon([A, B], [[-1, 1] if opA == "N" else [1, -1], [1, -2] if opB == "N" else [-2, 1]])
                assert np.allclose(got, reg, rtol=1e-12, atol=1e-12 * np.abs(reg).max()), (opA, opB, m, n, k)
        # device memory free after each round of calls (the first call on the
        # device may load the module that holds the static scratch array)
        free.append(torch.cuda.mem_get_info()[0])
    # no allocation by the entry point: a further round of calls leaves the
    # device's free memory exactly where it was
    for opA, opB, m, n, k, A, B, dA, dB, dC in inputs:
        assert gemm(opA.encode(), opB.encode(), m, n, k, 1.0, dA.data_ptr(), A.shape[0], dB.data_ptr(), B.shape[0],
                    0.0, dC.data_ptr(), m, ct.c_void_p(stream)) == IPEPS_OK
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free[-1]


def test_noalloc_gemm_rejects_shapes_beyond_the_grid(pkg):
    torch = _torch_cuda()
    lib = ct.CDLL(pkg.LIB_PATH)
    gemm = _noalloc(lib)
    # n = 65535*64 + 1 columns exceed the kernel grid: rejected on the host,
    # before any launch, so the one-element buffers are never read
    m, n, k = 1, 65535 * 64 + 1, 1
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    p = dummy.data_ptr()
    assert gemm(b"N", b"N", m, n, k, 1.0, p, m, p, k, 0.0, p, m, None) == IPEPS_EINVAL
