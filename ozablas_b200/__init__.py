"""ozablas_b200 -- B200-native Ozaki Scheme I / II FP64 GEMM.

Python mirror of the OzaBLAS operator interface (IlyaNyrkov/ozablas:
include/ozablas/ozablas.hpp:20,31, core/executor.hpp, core/workspace.hpp)
over the C ABI of include/oza_capi.h, loaded from the in-tree
``liboza_b200.so``.  The arithmetic runs only in the sm_100a kernels of that
library; there is no CPU fallback, and every entry point raises if the
library or a B200 is missing.

Matrices are row-major FP64 device buffers, passed either as raw device
pointers (int) or as contiguous CUDA ``torch.float64`` tensors.

    ex = CudaExecutor(0)
    ws = WorkspaceScheme2(ex, M, N, K, slices=16)
    ozaki_scheme2_gemm(ws, A, B, C)            # asynchronous
    t = OzaTimings(); ozaki_scheme2_gemm(ws, A, B, C, t)   # synchronous, per-step ms
"""
from __future__ import annotations

import ctypes
import os
import re
from dataclasses import dataclass

__all__ = [
    "LIB_PATH", "OzaError", "OzaTimeoutError", "OzaTimings", "CudaExecutor", "CpuExecutor",
    "WorkspaceScheme1", "WorkspaceScheme2", "ozaki_scheme1_gemm", "ozaki_scheme2_gemm",
    "generate_matrix", "scheme1_beta", "scheme2_k_param", "lib", "exported_symbols", "block_error",
    "autotune_slices", "autotune_scheme", "GroupGemm", "Server", "slices_for_target", "scheme_for_target",
    "ozaki_gemm_host", "selftest_wait_timeout", "set_residue_slicer", "residue_slicer",
    "OZA_SLICER_AUTO", "OZA_SLICER_TENSOR", "OZA_SLICER_CUDA_CORES",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboza_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "oza_capi.h")

OZA_OK, OZA_INVALID_ARG, OZA_OOM, OZA_CUDA_ERROR, OZA_TIMEOUT, OZA_UNSUPPORTED = range(6)
OZA_SCHEME1, OZA_SCHEME2 = 1, 2
OZA_WS_MATERIALIZE = 0x1
OZA_WS_REFERENCE_LAYOUT = 0x2
OZA_GROUP_NO_GRAPH = 0x2
BUF_SHIFT_A, BUF_SHIFT_B, BUF_A_SLICES, BUF_B_SLICES, BUF_C_TC = range(5)


class OzaError(RuntimeError):
    """CUDA failure or unsupported request (std::runtime_error in the C++ API)."""


class OzaTimeoutError(OzaError):
    """A bounded device-side wait expired inside a kernel."""


class _Timings(ctypes.Structure):
    _fields_ = [("step1_ms", ctypes.c_float), ("step2_ms", ctypes.c_float), ("step3_ms", ctypes.c_float),
                ("step4_ms", ctypes.c_float), ("total_ms", ctypes.c_float)]


class _WsInfo(ctypes.Structure):
    _fields_ = [("scheme", ctypes.c_int), ("slices", ctypes.c_int),
                ("M", ctypes.c_size_t), ("N", ctypes.c_size_t), ("K", ctypes.c_size_t),
                ("Mp", ctypes.c_size_t), ("Np", ctypes.c_size_t), ("Kp", ctypes.c_size_t),
                ("groups", ctypes.c_int), ("k_param", ctypes.c_int), ("beta", ctypes.c_int),
                ("flags", ctypes.c_uint), ("bytes", ctypes.c_size_t)]


class _GemmConfig(ctypes.Structure):
    _fields_ = [("band", ctypes.c_int), ("wait_hint_ns", ctypes.c_int), ("overlap_chunks", ctypes.c_int)]


class _GroupInfo(ctypes.Structure):
    _fields_ = [("count", ctypes.c_size_t), ("units", ctypes.c_size_t), ("bytes", ctypes.c_size_t),
                ("launches", ctypes.c_int), ("graph", ctypes.c_int)]


class _ServerConfig(ctypes.Structure):
    _fields_ = [("workspace_budget", ctypes.c_size_t), ("max_inflight", ctypes.c_int), ("max_batch", ctypes.c_int)]


class _RequestStats(ctypes.Structure):
    _fields_ = [("submit_s", ctypes.c_double), ("admit_s", ctypes.c_double), ("done_s", ctypes.c_double),
                ("slices", ctypes.c_int), ("batch_size", ctypes.c_int), ("status", ctypes.c_int),
                ("workspace_bytes", ctypes.c_size_t)]


class _ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_size_t), ("admitted", ctypes.c_size_t), ("completed", ctypes.c_size_t),
                ("queued", ctypes.c_size_t), ("batches", ctypes.c_size_t), ("max_batch_seen", ctypes.c_int),
                ("arena_used", ctypes.c_size_t), ("arena_peak", ctypes.c_size_t),
                ("workspace_budget", ctypes.c_size_t)]


@dataclass
class OzaTimings:
    """Per-step device milliseconds (reference: struct OzaTimings, workspace.hpp:97-103)."""
    step1_ms: float = 0.0
    step2_ms: float = 0.0
    step3_ms: float = 0.0
    step4_ms: float = 0.0
    total_ms: float = 0.0


_lib = None


def lib() -> ctypes.CDLL:
    """The loaded C-ABI library; raises OSError if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is missing: build it with `make -C ozablas_b200/csrc` "
                      "(or __graft_entry__.build()); there is no fallback implementation")
    L = ctypes.CDLL(LIB_PATH)
    P, S, I, U = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_uint
    sig = {
        "oza_last_error_string": (ctypes.c_char_p, []),
        "oza_version": (ctypes.c_char_p, []),
        "oza_executor_create": (I, [I, ctypes.POINTER(P)]),
        "oza_executor_destroy": (I, [P]),
        "oza_executor_alloc": (I, [P, ctypes.POINTER(P), S]),
        "oza_executor_free": (I, [P, P]),
        "oza_executor_copy": (I, [P, P, P, S, I]),
        "oza_executor_synchronize": (I, [P]),
        "oza_executor_set_stream": (I, [P, P]),
        "oza_executor_device": (I, [P, ctypes.POINTER(I)]),
        "oza_executor_blas_handle": (P, [P]),
        "oza_ws_create": (I, [P, I, S, S, S, I, U, ctypes.POINTER(P)]),
        "oza_ws_destroy": (I, [P]),
        "oza_ws_get_ptr": (I, [P, I, ctypes.POINTER(P)]),
        "oza_ws_get_info": (I, [P, ctypes.POINTER(_WsInfo)]),
        "oza_gemm": (I, [P, P, P, P, ctypes.POINTER(_Timings)]),
        "oza_gemm_host": (I, [P, P, P, P, ctypes.POINTER(_Timings)]),
        "oza_selftest_wait_timeout": (I, [P, ctypes.c_double, ctypes.POINTER(I), ctypes.POINTER(ctypes.c_double)]),
        "oza_ws_set_gemm_config": (I, [P, ctypes.POINTER(_GemmConfig)]),
        "oza_ws_get_gemm_config": (I, [P, ctypes.POINTER(_GemmConfig)]),
        "oza_autotune_gemm": (I, [P, P, P, P, ctypes.POINTER(_GemmConfig), ctypes.POINTER(ctypes.c_float)]),
        "oza_ws_device_error": (I, [P, ctypes.POINTER(I)]),
        "oza_generate_matrix": (I, [I, I, ctypes.c_double, I, P]),
        "oza_scheme1_beta": (I, [S]),
        "oza_block_error": (I, [P, P, P, P, S, S, S, I, U, ctypes.POINTER(ctypes.c_double)]),
        "oza_autotune_slices": (I, [P, I, S, S, S, P, P, ctypes.c_double, I, U, ctypes.POINTER(I),
                                    ctypes.POINTER(ctypes.c_double)]),
        "oza_scheme2_k_param": (I, [I, S]),
        "oza_group_create": (I, [P, I, S, ctypes.POINTER(S), ctypes.POINTER(S), ctypes.POINTER(S),
                                 ctypes.POINTER(I), U, ctypes.POINTER(P)]),
        "oza_group_destroy": (I, [P]),
        "oza_group_gemm": (I, [P, ctypes.POINTER(P), ctypes.POINTER(P), ctypes.POINTER(P),
                               ctypes.POINTER(_Timings)]),
        "oza_group_get_info": (I, [P, ctypes.POINTER(_GroupInfo)]),
        "oza_group_device_error": (I, [P, ctypes.POINTER(I)]),
        "oza_server_create": (I, [P, ctypes.POINTER(_ServerConfig), ctypes.POINTER(P)]),
        "oza_server_destroy": (I, [P]),
        "oza_server_submit": (I, [P, I, S, S, S, P, P, P, I, ctypes.POINTER(ctypes.c_uint64)]),
        "oza_server_wait": (I, [P, ctypes.c_uint64, ctypes.c_double, ctypes.POINTER(_RequestStats)]),
        "oza_server_get_stats": (I, [P, ctypes.POINTER(_ServerStats)]),
        "oza_server_request_bytes": (S, [I, S, S, S, I]),
        "oza_slices_for_target": (I, [ctypes.c_double, S, ctypes.c_double]),
        "oza_scheme_for_target": (I, [ctypes.c_double, S, ctypes.c_double, ctypes.POINTER(I)]),
        "oza_autotune_scheme": (I, [P, S, S, S, P, P, ctypes.c_double, I, U, ctypes.POINTER(I), ctypes.POINTER(I),
                                    ctypes.POINTER(ctypes.c_double)]),
        "oza_autotune_scheme_like": (I, [P, S, S, S, P, P, P, ctypes.c_double, I, U, ctypes.POINTER(I),
                                         ctypes.POINTER(I), ctypes.POINTER(ctypes.c_double)]),
        "oza_estimate_phi": (I, [P, S, S, S, P, P, I, U, ctypes.POINTER(ctypes.c_double)]),
        "oza_set_residue_slicer": (I, [I]),
        "oza_get_residue_slicer": (I, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype, fn.argtypes = res, args
    _lib = L
    return L


def exported_symbols() -> list[str]:
    """Every function name declared in include/oza_capi.h."""
    with open(HEADER_PATH) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(oza_[a-z0-9_]+)\s*\(", text)))


def _check(status: int) -> None:
    if status == OZA_OK:
        return
    msg = (lib().oza_last_error_string() or b"").decode(errors="replace")
    if status == OZA_INVALID_ARG:
        raise ValueError(msg)
    if status == OZA_OOM:
        raise MemoryError(msg)
    if status == OZA_TIMEOUT:
        raise OzaTimeoutError(msg)
    raise OzaError(msg)


def _ptr(x) -> int:
    """Device address of an int or of a contiguous CUDA float64 torch tensor."""
    if x is None:
        return 0
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        if not x.is_cuda:
            raise ValueError("matrix must live on the GPU (no CPU fallback)")
        if not x.is_contiguous():
            raise ValueError("matrix must be contiguous (row-major)")
        return int(x.data_ptr())
    raise TypeError(f"expected a device pointer or a CUDA tensor, got {type(x).__name__}")


class CpuExecutor:
    """Host executor kept for API compatibility; the GEMMs reject it, as the
    reference's dispatcher does (src/ozablas.cpp:42-45)."""


class CudaExecutor:
    """Device, stream and allocations (reference CudaExecutor, executor.cpp:61-114)."""

    def __init__(self, device_id: int = 0):
        h = ctypes.c_void_p()
        _check(lib().oza_executor_create(int(device_id), ctypes.byref(h)))
        self._h = h
        self.device_id = int(device_id)

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def allocate(self, nbytes: int) -> int:
        p = ctypes.c_void_p()
        _check(lib().oza_executor_alloc(self._h, ctypes.byref(p), int(nbytes)))
        return int(p.value or 0)

    def free(self, ptr: int) -> None:
        _check(lib().oza_executor_free(self._h, ctypes.c_void_p(ptr)))

    def copy_from_host(self, dst: int, src: int, nbytes: int) -> None:
        _check(lib().oza_executor_copy(self._h, ctypes.c_void_p(dst), ctypes.c_void_p(src), int(nbytes), 1))

    def copy_to_host(self, dst: int, src: int, nbytes: int) -> None:
        _check(lib().oza_executor_copy(self._h, ctypes.c_void_p(dst), ctypes.c_void_p(src), int(nbytes), 2))

    def copy_device_to_device(self, dst: int, src: int, nbytes: int) -> None:
        _check(lib().oza_executor_copy(self._h, ctypes.c_void_p(dst), ctypes.c_void_p(src), int(nbytes), 3))

    def synchronize(self) -> None:
        _check(lib().oza_executor_synchronize(self._h))

    def set_stream(self, stream) -> None:
        """Issue subsequent work on a CUDA stream (int handle, torch.cuda.Stream, or None)."""
        s = getattr(stream, "cuda_stream", stream)
        _check(lib().oza_executor_set_stream(self._h, ctypes.c_void_p(int(s or 0))))

    def get_blas_handle(self) -> int:
        return int(lib().oza_executor_blas_handle(self._h) or 0)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.oza_executor_destroy(h)
            self._h = None


class _Workspace:
    _scheme = 0

    def __init__(self, executor, M: int, N: int, K: int, slices: int, materialize: bool = False,
                 reference_layout: bool = False):
        if executor is None:
            raise ValueError("OzaBLAS: Executor cannot be null.")
        if not isinstance(executor, CudaExecutor):
            raise OzaError("OzaBLAS: No suitable hardware backend found for the provided Executor.")
        self._exec = executor   # keeps the executor alive, like the reference's shared_ptr
        h = ctypes.c_void_p()
        flags = (OZA_WS_MATERIALIZE if materialize else 0) | (OZA_WS_REFERENCE_LAYOUT if reference_layout else 0)
        _check(lib().oza_ws_create(executor.handle, self._scheme, int(M), int(N), int(K), int(slices),
                                   flags, ctypes.byref(h)))
        self._h = h
        info = _WsInfo()
        _check(lib().oza_ws_get_info(h, ctypes.byref(info)))
        self.info = {f: getattr(info, f) for f, _ in _WsInfo._fields_}

    @property
    def handle(self):
        return self._h

    def get_executor(self):
        return self._exec

    def get_M(self): return self.info["M"]
    def get_N(self): return self.info["N"]
    def get_K(self): return self.info["K"]
    def get_slices(self): return self.info["slices"]
    def get_Mp(self): return self.info["Mp"]
    def get_Np(self): return self.info["Np"]
    def get_Kp(self): return self.info["Kp"]

    def _buf(self, which: int) -> int:
        p = ctypes.c_void_p()
        _check(lib().oza_ws_get_ptr(self._h, which, ctypes.byref(p)))
        return int(p.value or 0)

    def get_shift_A(self): return self._buf(BUF_SHIFT_A)
    def get_shift_B(self): return self._buf(BUF_SHIFT_B)
    def get_A_slices(self): return self._buf(BUF_A_SLICES)
    def get_B_slices(self): return self._buf(BUF_B_SLICES)
    def get_C_tc(self): return self._buf(BUF_C_TC)

    def device_error(self) -> int:
        c = ctypes.c_int()
        _check(lib().oza_ws_device_error(self._h, ctypes.byref(c)))
        return c.value

    def set_gemm_config(self, band: int = 0, wait_hint_ns: int = 0, overlap_chunks: int = 0) -> None:
        """Step-3 kernel configuration; results are bit-identical whatever it is
        (extension: oza_ws_set_gemm_config).

        band           m-tiles (128 rows each) per rasterisation band (0: 16)
        wait_hint_ns   suspend-time hint of the kernel's mbarrier waits (0: poll)
        overlap_chunks Scheme II fused path without timings: >= 2 overlaps A's
                       slicing and the reconstruction with the GEMM in that many
                       row chunks; 1 runs the steps in order; 0 takes 2 chunks
                       for 8 to 47 row tiles of 128, else 1."""
        cfg = _GemmConfig(int(band), int(wait_hint_ns), int(overlap_chunks))
        _check(lib().oza_ws_set_gemm_config(self._h, ctypes.byref(cfg)))

    def get_gemm_config(self) -> dict:
        cfg = _GemmConfig()
        _check(lib().oza_ws_get_gemm_config(self._h, ctypes.byref(cfg)))
        return {f: getattr(cfg, f) for f, _ in _GemmConfig._fields_}

    def autotune_gemm(self, A, B, C):
        """Time every step-3 configuration on these inputs, keep the fastest;
        returns (config dict, step-3 ms).  C is overwritten."""
        cfg = _GemmConfig()
        ms = ctypes.c_float()
        _check(lib().oza_autotune_gemm(self._h, ctypes.c_void_p(_ptr(A)), ctypes.c_void_p(_ptr(B)),
                                       ctypes.c_void_p(_ptr(C)), ctypes.byref(cfg), ctypes.byref(ms)))
        return {f: getattr(cfg, f) for f, _ in _GemmConfig._fields_}, ms.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.oza_ws_destroy(h)
            self._h = None


class WorkspaceScheme1(_Workspace):
    """Scheme I workspace (reference WorkspaceScheme1, workspace.cpp:21-56); slices >= 1."""
    _scheme = OZA_SCHEME1


class WorkspaceScheme2(_Workspace):
    """Scheme II workspace (reference WorkspaceScheme2, workspace.cpp:63-126); 1 <= slices <= 20."""
    _scheme = OZA_SCHEME2


def _gemm(ws, A, B, C, timings):
    t = _Timings() if timings is not None else None
    _check(lib().oza_gemm(ws.handle, ctypes.c_void_p(_ptr(A)), ctypes.c_void_p(_ptr(B)),
                          ctypes.c_void_p(_ptr(C)), ctypes.byref(t) if t is not None else None))
    if timings is not None:
        for f, _ in _Timings._fields_:
            setattr(timings, f, float(getattr(t, f)))


def _check_shapes(ws, A, B, C):
    if hasattr(A, "shape") and hasattr(B, "shape") and hasattr(C, "shape"):
        M, N, K = ws.get_M(), ws.get_N(), ws.get_K()
        if tuple(A.shape) != (M, K) or tuple(B.shape) != (K, N) or tuple(C.shape) != (M, N):
            raise ValueError(f"shapes {tuple(A.shape)} x {tuple(B.shape)} -> {tuple(C.shape)} "
                             f"do not match the workspace ({M}x{K} x {K}x{N})")
        for t in (A, B, C):
            if str(getattr(t, "dtype", "torch.float64")) != "torch.float64":
                raise ValueError("matrices must be float64")


def ozaki_scheme1_gemm(ws: WorkspaceScheme1, A, B, C, timings: OzaTimings | None = None) -> None:
    """C = A * B by Ozaki Scheme I (reference ozaki_scheme1_gemm, ozablas.hpp:20)."""
    if not isinstance(ws, WorkspaceScheme1):
        raise TypeError("ozaki_scheme1_gemm needs a WorkspaceScheme1")
    _check_shapes(ws, A, B, C)
    _gemm(ws, A, B, C, timings)


def ozaki_scheme2_gemm(ws: WorkspaceScheme2, A, B, C, timings: OzaTimings | None = None) -> None:
    """C = A * B by Ozaki Scheme II (reference ozaki_scheme2_gemm, ozablas.hpp:31)."""
    if not isinstance(ws, WorkspaceScheme2):
        raise TypeError("ozaki_scheme2_gemm needs a WorkspaceScheme2")
    _check_shapes(ws, A, B, C)
    _gemm(ws, A, B, C, timings)


class GroupGemm:
    """Many independent Scheme II FP64 GEMMs of different shapes, run as one
    launch per stage and replayed from a CUDA graph (extension; the reference
    runs one GEMM per call).

        g = GroupGemm(ex, [(M0, N0, K0), (M1, N1, K1), ...], slices=16)
        g(As, Bs, Cs)     # lists of device matrices, asynchronous
    """

    def __init__(self, executor, shapes, slices, graph: bool = True):
        if not isinstance(executor, CudaExecutor):
            raise OzaError("OzaBLAS: No suitable hardware backend found for the provided Executor.")
        self._exec = executor
        shapes = [tuple(int(x) for x in s) for s in shapes]
        n = len(shapes)
        if isinstance(slices, int):
            slices = [slices] * n
        if len(slices) != n:
            raise ValueError("one slice count per problem")
        self.shapes = shapes
        self.slices = [int(s) for s in slices]
        arr = ctypes.c_size_t * n
        Ms, Ns, Ks = arr(*[s[0] for s in shapes]), arr(*[s[1] for s in shapes]), arr(*[s[2] for s in shapes])
        Ss = (ctypes.c_int * n)(*self.slices)
        h = ctypes.c_void_p()
        _check(lib().oza_group_create(executor.handle, OZA_SCHEME2, n, Ms, Ns, Ks, Ss,
                                      0 if graph else OZA_GROUP_NO_GRAPH, ctypes.byref(h)))
        self._h = h
        info = _GroupInfo()
        _check(lib().oza_group_get_info(h, ctypes.byref(info)))
        self.info = {f: getattr(info, f) for f, _ in _GroupInfo._fields_}
        self._parr = ctypes.c_void_p * n

    def __call__(self, As, Bs, Cs, timings: OzaTimings | None = None) -> None:
        n = len(self.shapes)
        if not (len(As) == len(Bs) == len(Cs) == n):
            raise ValueError(f"expected {n} matrices of each operand")
        for (M, N, K), A, B, C in zip(self.shapes, As, Bs, Cs):
            if hasattr(A, "shape") and (tuple(A.shape) != (M, K) or tuple(B.shape) != (K, N)
                                        or tuple(C.shape) != (M, N)):
                raise ValueError(f"shapes do not match problem {(M, N, K)}")
        pa = self._parr(*[_ptr(a) for a in As])
        pb = self._parr(*[_ptr(b) for b in Bs])
        pc = self._parr(*[_ptr(c) for c in Cs])
        t = _Timings() if timings is not None else None
        _check(lib().oza_group_gemm(self._h, pa, pb, pc, ctypes.byref(t) if t is not None else None))
        if timings is not None:
            for f, _ in _Timings._fields_:
                setattr(timings, f, float(getattr(t, f)))

    def device_error(self) -> int:
        c = ctypes.c_int()
        _check(lib().oza_group_device_error(self._h, ctypes.byref(c)))
        return c.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.oza_group_destroy(h)
            self._h = None


class Server:
    """Request loop with continuous batching for FP64 GEMMs (extension; the
    reference has no request loop).  Requests are admitted in arrival order
    while their workspaces fit in `workspace_budget` bytes of device memory and
    one of `max_inflight` stream slots is free; the Scheme II requests of a
    batch run the grouped kernels, a Scheme I request runs on its own.

        srv = Server(ex, 8 << 30)
        rid = srv.submit(A, B, C, slices=16)   # device matrices, kept alive by the caller
        stats = srv.wait(rid)                  # timestamps in seconds since creation
    """

    def __init__(self, executor, workspace_budget: int, max_inflight: int = 2, max_batch: int = 64):
        if not isinstance(executor, CudaExecutor):
            raise OzaError("OzaBLAS: No suitable hardware backend found for the provided Executor.")
        self._exec = executor
        cfg = _ServerConfig(int(workspace_budget), int(max_inflight), int(max_batch))
        h = ctypes.c_void_p()
        _check(lib().oza_server_create(executor.handle, ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h

    @staticmethod
    def request_bytes(M: int, N: int, K: int, slices: int, scheme: int = OZA_SCHEME2) -> int:
        return int(lib().oza_server_request_bytes(int(scheme), int(M), int(N), int(K), int(slices)))

    def submit(self, A, B, C, slices: int, M: int | None = None, N: int | None = None,
               K: int | None = None, scheme: int = OZA_SCHEME2) -> int:
        """Queue C = A * B with `slices` slices/moduli of `scheme` (Scheme II
        requests are batched together; a Scheme I request runs on its own)."""
        if M is None:
            M, K = A.shape
            N = B.shape[1]
            if tuple(B.shape) != (K, N) or tuple(C.shape) != (M, N):
                raise ValueError("shapes do not agree")
        rid = ctypes.c_uint64()
        _check(lib().oza_server_submit(self._h, int(scheme), int(M), int(N), int(K), ctypes.c_void_p(_ptr(A)),
                                       ctypes.c_void_p(_ptr(B)), ctypes.c_void_p(_ptr(C)), int(slices),
                                       ctypes.byref(rid)))
        return rid.value

    def wait(self, rid: int, timeout: float | None = None) -> dict:
        st = _RequestStats()
        _check(lib().oza_server_wait(self._h, int(rid), -1.0 if timeout is None else float(timeout),
                                     ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in _RequestStats._fields_}

    def stats(self) -> dict:
        st = _ServerStats()
        _check(lib().oza_server_get_stats(self._h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in _ServerStats._fields_}

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.oza_server_destroy(h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        self.close()


def _host_ptr(x, shape, writable=False) -> int:
    """Address of a C-contiguous float64 host array (numpy or CPU torch tensor)."""
    if hasattr(x, "data_ptr"):
        if x.is_cuda:
            raise ValueError("host matrix expected (a CPU tensor or numpy array)")
        if not x.is_contiguous() or str(x.dtype) != "torch.float64":
            raise ValueError("host matrices must be contiguous float64")
        if tuple(x.shape) != tuple(shape):
            raise ValueError(f"shape {tuple(x.shape)} does not match {tuple(shape)}")
        return int(x.data_ptr())
    import numpy as np
    if not isinstance(x, np.ndarray) or x.dtype != np.float64 or not x.flags["C_CONTIGUOUS"]:
        raise ValueError("host matrices must be C-contiguous float64 numpy arrays or CPU tensors")
    if writable and not x.flags["WRITEABLE"]:
        raise ValueError("output array is read-only")
    if tuple(x.shape) != tuple(shape):
        raise ValueError(f"shape {tuple(x.shape)} does not match {tuple(shape)}")
    return int(x.ctypes.data)


def ozaki_gemm_host(ws, A, B, C, timings: OzaTimings | None = None) -> None:
    """C = A * B with host matrices (pinned CPU tensors overlap the copies with
    the compute), synchronous; bit-identical to the device-buffer call
    (extension: oza_gemm_host)."""
    M, N, K = ws.get_M(), ws.get_N(), ws.get_K()
    t = _Timings() if timings is not None else None
    _check(lib().oza_gemm_host(ws.handle, ctypes.c_void_p(_host_ptr(A, (M, K))),
                               ctypes.c_void_p(_host_ptr(B, (K, N))),
                               ctypes.c_void_p(_host_ptr(C, (M, N), writable=True)),
                               ctypes.byref(t) if t is not None else None))
    if timings is not None:
        for f, _ in _Timings._fields_:
            setattr(timings, f, float(getattr(t, f)))


OZA_SLICER_AUTO, OZA_SLICER_CUDA_CORES, OZA_SLICER_TENSOR = 0, 1, 2


def set_residue_slicer(mode: int) -> None:
    """Process-wide Scheme II step-2 slicer: OZA_SLICER_AUTO (default; tcgen05
    digit products from S = 12 to 16, dp4a below), OZA_SLICER_TENSOR (tcgen05
    for every S <= 16) or OZA_SLICER_CUDA_CORES (dp4a).  All give identical
    residue planes."""
    _check(lib().oza_set_residue_slicer(int(mode)))


def residue_slicer() -> int:
    return int(lib().oza_get_residue_slicer())


def selftest_wait_timeout(executor, limit_s: float = 0.2):
    """Run one bounded device wait that nothing satisfies; returns (device
    error code, kernel seconds).  Code 1 means the wait expired and reported."""
    code = ctypes.c_int()
    el = ctypes.c_double()
    _check(lib().oza_selftest_wait_timeout(executor.handle, float(limit_s), ctypes.byref(code), ctypes.byref(el)))
    return code.value, el.value


def generate_matrix(rows: int, cols: int, phi: float = 0.5, seed: int = 42):
    """Seeded (U-0.5)*exp(phi*N(0,1)) matrix as a numpy array (reference
    generate_ozaki_matrix, utils/matrix_gen.hpp:15-34)."""
    import numpy as np
    out = np.empty((rows, cols), dtype=np.float64)
    _check(lib().oza_generate_matrix(int(rows), int(cols), float(phi), int(seed),
                                     out.ctypes.data_as(ctypes.c_void_p)))
    return out


def block_error(executor, A, B, C, M: int, N: int, K: int, block: int = 96, seed: int = 7) -> float:
    """Max relative error of C against a double-double reference on a seeded
    block of `block` rows x `block` columns (device matrices)."""
    e = ctypes.c_double()
    _check(lib().oza_block_error(executor.handle, ctypes.c_void_p(_ptr(A)), ctypes.c_void_p(_ptr(B)),
                                 ctypes.c_void_p(_ptr(C)), int(M), int(N), int(K), int(block), int(seed),
                                 ctypes.byref(e)))
    return e.value


def autotune_slices(executor, scheme: int, A, B, M: int, N: int, K: int, target_rel_err: float,
                    block: int = 96, seed: int = 7):
    """Smallest slice count meeting target_rel_err on a sampled block; returns
    (slices, sampled error).  Raises OzaError if 20 slices miss the target."""
    s = ctypes.c_int()
    e = ctypes.c_double()
    _check(lib().oza_autotune_slices(executor.handle, int(scheme), int(M), int(N), int(K),
                                     ctypes.c_void_p(_ptr(A)), ctypes.c_void_p(_ptr(B)), float(target_rel_err),
                                     int(block), int(seed), ctypes.byref(s), ctypes.byref(e)))
    return s.value, e.value


def autotune_scheme(executor, A, B, M: int, N: int, K: int, target_rel_err: float, block: int = 96,
                    seed: int = 7):
    """Scheme and slice count meeting target_rel_err with the fewest INT8 GEMMs
    on two independent sampled blocks (Scheme I where Scheme II's 20 moduli
    miss it); returns (scheme, slices, largest sampled error).  Raises OzaError
    if neither scheme reaches it."""
    sc, s = ctypes.c_int(), ctypes.c_int()
    e = ctypes.c_double()
    _check(lib().oza_autotune_scheme(executor.handle, int(M), int(N), int(K), ctypes.c_void_p(_ptr(A)),
                                     ctypes.c_void_p(_ptr(B)), float(target_rel_err), int(block), int(seed),
                                     ctypes.byref(sc), ctypes.byref(s), ctypes.byref(e)))
    return sc.value, s.value, e.value


def autotune_scheme_like(executor, A, B, M: int, N: int, K: int, C_ref, factor: float = 1.0, block: int = 96,
                         seed: int = 7):
    """Scheme and slice count whose error is at most factor times C_ref's
    (another result of A @ B, e.g. native DGEMM's) on every sampled block, with
    the fewest INT8 GEMMs; returns (scheme, slices, largest sampled error
    ratio).  Raises OzaError if neither scheme reaches it."""
    sc, s = ctypes.c_int(), ctypes.c_int()
    e = ctypes.c_double()
    _check(lib().oza_autotune_scheme_like(executor.handle, int(M), int(N), int(K), ctypes.c_void_p(_ptr(A)),
                                          ctypes.c_void_p(_ptr(B)), ctypes.c_void_p(_ptr(C_ref)), float(factor),
                                          int(block), int(seed), ctypes.byref(sc), ctypes.byref(s), ctypes.byref(e)))
    return sc.value, s.value, e.value


def estimate_phi(executor, A, B, M: int, N: int, K: int, block: int = 96, seed: int = 7) -> float:
    """The exponent spread phi of the calibrated tables, estimated from
    sampled rows of A and columns of B (device matrices)."""
    phi = ctypes.c_double()
    _check(lib().oza_estimate_phi(executor.handle, int(M), int(N), int(K), ctypes.c_void_p(_ptr(A)),
                                  ctypes.c_void_p(_ptr(B)), int(block), int(seed), ctypes.byref(phi)))
    return phi.value


def scheme_for_target(target_rel_err: float, K: int, phi: float = 2.0):
    """(scheme, slices) for a maximum-relative-error target from the calibrated
    tables (no GPU work): the scheme reaching it with fewer INT8 GEMMs; slices
    21 means neither reaches it with 20."""
    s = ctypes.c_int()
    sc = int(lib().oza_scheme_for_target(float(target_rel_err), int(K), float(phi), ctypes.byref(s)))
    if sc == 0:
        raise ValueError("target must be > 0, K >= 1, phi >= 0")
    return sc, s.value


def slices_for_target(target_rel_err: float, K: int, phi: float = 2.0) -> int:
    """Scheme II slice count for a maximum-relative-error target from the
    calibrated table (no GPU work); 21 means 20 slices did not reach it."""
    s = int(lib().oza_slices_for_target(float(target_rel_err), int(K), float(phi)))
    if s == 0:
        raise ValueError("target must be > 0, K >= 1, phi >= 0")
    return s


def scheme1_beta(K: int) -> int:
    return int(lib().oza_scheme1_beta(int(K)))


def scheme2_k_param(slices: int, K: int) -> int:
    return int(lib().oza_scheme2_k_param(int(slices), int(K)))
