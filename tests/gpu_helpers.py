"""Helpers for the GPU parity tests: run the sm_100a pipeline through the C ABI
and read every intermediate back in the reference's layouts."""
import ctypes

import numpy as np


def run_pipeline(oz, executor, scheme, A, B, S, materialize=True):
    import torch
    M, K = A.shape
    N = B.shape[1]
    ws_cls = oz.WorkspaceScheme2 if scheme == 2 else oz.WorkspaceScheme1
    fn = oz.ozaki_scheme2_gemm if scheme == 2 else oz.ozaki_scheme1_gemm
    ws = ws_cls(executor, M, N, K, S, materialize=materialize)
    dA = torch.from_numpy(np.ascontiguousarray(A)).cuda()
    dB = torch.from_numpy(np.ascontiguousarray(B)).cuda()
    dC = torch.full((M, N), float("nan"), dtype=torch.float64, device="cuda")
    t = oz.OzaTimings()
    fn(ws, dA, dB, dC, t)
    out = dict(C=dC.cpu().numpy(), timings=t, ws=ws)
    out.update(read_intermediates(executor, ws))
    return out


def _read(executor, ptr, shape, dtype):
    a = np.empty(shape, dtype)
    executor.copy_to_host(a.ctypes.data_as(ctypes.c_void_p).value, ptr, a.nbytes)
    return a


def read_intermediates(executor, ws):
    """Workspace buffers in the reference layouts: slices [S][M][K] and
    [S][K][N], INT32 products [G][M][N]; also the raw padded planes."""
    i = ws.info
    M, N, K, Mp, Np, Kp, S, G = i["M"], i["N"], i["K"], i["Mp"], i["Np"], i["Kp"], i["slices"], i["groups"]
    sA = _read(executor, ws.get_shift_A(), (M,), np.int32)
    sB = _read(executor, ws.get_shift_B(), (N,), np.int32)
    Ap = _read(executor, ws.get_A_slices(), (S, Mp, Kp), np.int8)
    Bp = _read(executor, ws.get_B_slices(), (S, Np, Kp), np.int8)
    out = dict(shift_A=sA, shift_B=sB, A_slices=Ap[:, :M, :K], B_slices=Bp[:, :N, :K].transpose(0, 2, 1),
               A_planes=Ap, B_planes=Bp)
    if ws.get_C_tc():   # absent when Scheme II runs the CRT inside the GEMM epilogue
        Cp = _read(executor, ws.get_C_tc(), (G, Mp, Np), np.int32)
        out.update(C_tc=Cp[:, :M, :N], C_planes=Cp)
    return out


def bits(x):
    return np.ascontiguousarray(x, np.float64).view(np.int64)
