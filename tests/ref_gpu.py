"""ctypes wrapper of baseline/_ref/libozablas_ref_gpu.so: the reference's own
cuBLAS-backed GPU pipeline (IlyaNyrkov/ozablas src/cuda/pipeline.cu) driven
through its public C++ API.  Used by the GPU tests as a second parity pin."""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SO = os.path.join(ROOT, "baseline", "_ref", "libozablas_ref_gpu.so")


def available():
    return os.path.exists(SO)


_L = None


def lib():
    global _L
    if _L is None:
        L = ctypes.CDLL(SO)
        L.refgpu_init.argtypes = [ctypes.c_int]
        L.refgpu_ws_create.restype = ctypes.c_void_p
        L.refgpu_ws_create.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_int]
        L.refgpu_ws_destroy.argtypes = [ctypes.c_void_p]
        L.refgpu_ws_ptr.restype = ctypes.c_void_p
        L.refgpu_ws_ptr.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.refgpu_gemm.argtypes = [ctypes.c_void_p] * 5
        L.refgpu_dgemm.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int] * 3
        assert L.refgpu_init(0) == 0
        _L = L
    return _L


def run(executor, scheme, A, B, S):
    """Reference pipeline on the GPU.  Returns C and the intermediates in the
    reference's layouts (Scheme I C_tc holds only the last group, g = S + 1)."""
    import torch
    L = lib()
    M, K = A.shape
    N = B.shape[1]
    h = L.refgpu_ws_create(scheme, M, N, K, S)
    assert h, "reference workspace allocation failed"
    try:
        dA = torch.from_numpy(np.ascontiguousarray(A)).cuda()
        dB = torch.from_numpy(np.ascontiguousarray(B)).cuda()
        dC = torch.empty(M, N, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        assert L.refgpu_gemm(h, dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), None) == 0
        torch.cuda.synchronize()

        def grab(which, count, dtype):
            a = np.empty(count, dtype)
            executor.copy_to_host(a.ctypes.data_as(ctypes.c_void_p).value, L.refgpu_ws_ptr(h, which), a.nbytes)
            return a

        out = dict(C=dC.cpu().numpy(),
                   shift_A=grab(0, M, np.int32), shift_B=grab(1, N, np.int32),
                   A_slices=grab(2, S * M * K, np.int8).reshape(S, M, K),
                   B_slices=grab(3, S * K * N, np.int8).reshape(S, K, N))
        G = S if scheme == 2 else 1
        out["C_tc"] = grab(4, G * M * N, np.int32).reshape(G, M, N)
        return out
    finally:
        L.refgpu_ws_destroy(h)


def run_device(executor, scheme, dA, dB, S):
    """The reference pipeline on device inputs (CUDA float64 tensors); returns
    C and the intermediates as CUDA tensors in the reference's layouts, copied
    out of its workspace before that is freed (for sizes where host copies
    would be slow)."""
    import torch
    L = lib()
    M, K = dA.shape
    N = dB.shape[1]
    h = L.refgpu_ws_create(scheme, M, N, K, S)
    assert h, "reference workspace allocation failed"
    try:
        dC = torch.empty(M, N, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        assert L.refgpu_gemm(h, dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), None) == 0
        torch.cuda.synchronize()

        def grab(which, shape, dtype):
            t = torch.empty(shape, dtype=dtype, device="cuda")
            executor.copy_device_to_device(t.data_ptr(), L.refgpu_ws_ptr(h, which), t.numel() * t.element_size())
            return t

        G = S if scheme == 2 else 1
        return dict(C=dC, shift_A=grab(0, (M,), torch.int32), shift_B=grab(1, (N,), torch.int32),
                    A_slices=grab(2, (S, M, K), torch.int8), B_slices=grab(3, (S, K, N), torch.int8),
                    C_tc=grab(4, (G, M, N), torch.int32))
    finally:
        L.refgpu_ws_destroy(h)
