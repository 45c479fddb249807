"""oracle -- CPU parity checkers for the Ozaki Scheme I / II pipeline.

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by
bench.py's CPU-baseline leg, always as the checker, never as the product.

Two libraries, both built by oracle/Makefile:
  * ``liboza_oracle.so`` -- this repository's C restatement of the reference
    algorithm (oza_oracle.c), functions prefixed ``oo_``;
  * ``_ref/libozaref_cpu.so`` -- the reference's own kernel source
    (src/pipeline/*.hpp of IlyaNyrkov/ozablas) compiled for the host through
    ref_shim.cpp, functions prefixed ``ref_`` (present only where the
    reference tree was available at build time).

All arrays are numpy, row-major; slice/residue planes use the reference layout
[S][rows][cols].
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(_HERE, "liboza_oracle.so")
REF_CPU_SO = os.path.join(_HERE, "_ref", "libozaref_cpu.so")
REF_GPU_SO = os.path.join(_HERE, "_ref", "libozablas_ref_gpu.so")

_P = ctypes.c_void_p
_L = ctypes.c_long
_I = ctypes.c_int


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


class _Lazy:
    def __init__(self, path, sigs):
        self.path, self.sigs, self.L = path, sigs, None

    def available(self):
        return os.path.exists(self.path)

    def __getattr__(self, name):
        if self.L is None:
            if not os.path.exists(self.path):
                raise OSError(f"{self.path} not built (make -C oracle)")
            L = ctypes.CDLL(self.path)
            for n, (res, args) in self.sigs.items():
                f = getattr(L, n)
                f.restype, f.argtypes = res, args
            self.L = L
        return getattr(self.L, name)


_oo = _Lazy(ORACLE_SO, {
    "oo_crt_tables": (None, [_I, _P, _P, _P, _P]),
    "oo_modulus": (ctypes.c_uint, [_I]),
    "oo_crt_M_double": (ctypes.c_double, [_I]),
    "oo_scheme1_beta": (_I, [_L]),
    "oo_scheme2_kparam": (_I, [_I, _L]),
    "oo_row_shifts": (None, [_P, _L, _L, _I, _P]),
    "oo_col_shifts": (None, [_P, _L, _L, _I, _P]),
    "oo_slice2": (None, [_P, _L, _L, _P, _I, _I, _P]),
    "oo_slice1": (None, [_P, _L, _L, _P, _I, _I, _I, _P]),
    "oo_gemm_i8": (None, [_P, _P, _L, _L, _L, _P, _I]),
    "oo_reconstruct2": (None, [_P, _P, _P, _L, _L, _I, _P]),
    "oo_reconstruct1_group": (None, [_P, _P, _P, _L, _L, _I, _I, _P]),
    "oo_scheme2_gemm": (_I, [_P, _P, _L, _L, _L, _I, _P, _P, _P, _P, _P, _P]),
    "oo_scheme1_gemm": (_I, [_P, _P, _L, _L, _L, _I, _P, _P, _P, _P, _P, _P]),
    "oo_gemm_fp128": (None, [_P, _P, _L, _L, _L, _P]),
    "oo_gemm_fp128_sampled": (None, [_P, _P, _L, _L, _L, _P, _P, _L, _P]),
    "oo_gemm_dd": (None, [_P, _P, _L, _L, _L, _P]),
    "oo_gemm_f64": (None, [_P, _P, _L, _L, _L, _P]),
    "oo_num_threads": (_I, []),
})

_ref = _Lazy(REF_CPU_SO, {
    "ref_get_tables": (None, [_P, _P, _P, _P, _P]),
    "ref_scheme1_beta": (_I, [_I]),
    "ref_scheme2_kparam": (_I, [_I, _I]),
    "ref_row_shifts": (None, [_P, _I, _I, _I, _P]),
    "ref_col_shifts": (None, [_P, _I, _I, _I, _P]),
    "ref_slice2": (None, [_P, _I, _I, _P, _I, _I, _P]),
    "ref_slice1": (None, [_P, _I, _I, _P, _I, _I, _I, _P]),
    "ref_reconstruct2": (None, [_P, _P, _P, _I, _I, _I, _P]),
    "ref_reconstruct1_group": (None, [_P, _P, _P, _I, _I, _I, _I, _P]),
    "ref_cpu_scheme2_gemm": (None, [_P, _P, _P, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P]),
    "ref_cpu_scheme1_gemm": (None, [_P, _P, _P, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P]),
    "ref_generate_matrix": (None, [_I, _I, ctypes.c_double, _I, _P]),
})

MAX_SLICES = 20


def ref_available() -> bool:
    return _ref.available()


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ------------------------------------------------------------------ oracle (restatement)
class Oracle:
    """numpy front end of oza_oracle.c."""

    @staticmethod
    def moduli():
        return [int(_oo.oo_modulus(i)) for i in range(MAX_SLICES)]

    @staticmethod
    def crt_tables(S):
        M = np.zeros(4, np.uint64); Mh = np.zeros(4, np.uint64)
        P = np.zeros((MAX_SLICES, 4), np.uint64); I = np.zeros(MAX_SLICES, np.uint64)
        _oo.oo_crt_tables(S, _p(M), _p(Mh), _p(P), _p(I))
        return M, Mh, P[:S], I[:S]

    @staticmethod
    def beta(K):
        return int(_oo.oo_scheme1_beta(K))

    @staticmethod
    def k_param(S, K):
        return int(_oo.oo_scheme2_kparam(S, K))

    @staticmethod
    def row_shifts(A, offset):
        A = _f64(A); out = np.empty(A.shape[0], np.int32)
        _oo.oo_row_shifts(_p(A), A.shape[0], A.shape[1], offset, _p(out))
        return out

    @staticmethod
    def col_shifts(B, offset):
        B = _f64(B); out = np.empty(B.shape[1], np.int32)
        _oo.oo_col_shifts(_p(B), B.shape[0], B.shape[1], offset, _p(out))
        return out

    @staticmethod
    def slice2(X, shifts, per_row, S):
        X = _f64(X); sh = np.ascontiguousarray(shifts, np.int32)
        out = np.empty((S,) + X.shape, np.int8)
        _oo.oo_slice2(_p(X), X.shape[0], X.shape[1], _p(sh), int(per_row), S, _p(out))
        return out

    @staticmethod
    def slice1(X, neg_exp, per_row, S, beta):
        X = _f64(X); sh = np.ascontiguousarray(neg_exp, np.int32)
        out = np.empty((S,) + X.shape, np.int8)
        _oo.oo_slice1(_p(X), X.shape[0], X.shape[1], _p(sh), int(per_row), S, beta, _p(out))
        return out

    @staticmethod
    def gemm_i8(A, B, C=None):
        A = np.ascontiguousarray(A, np.int8); B = np.ascontiguousarray(B, np.int8)
        M, K = A.shape; N = B.shape[1]
        acc = C is not None
        out = np.ascontiguousarray(C, np.int32).copy() if acc else np.empty((M, N), np.int32)
        _oo.oo_gemm_i8(_p(A), _p(B), M, N, K, _p(out), int(acc))
        return out

    @staticmethod
    def reconstruct2(Ctc, sA, sB):
        Ctc = np.ascontiguousarray(Ctc, np.int32); S, M, N = Ctc.shape
        sA = np.ascontiguousarray(sA, np.int32); sB = np.ascontiguousarray(sB, np.int32)
        C = np.empty((M, N), np.float64)
        _oo.oo_reconstruct2(_p(Ctc), _p(sA), _p(sB), M, N, S, _p(C))
        return C

    @staticmethod
    def reconstruct1_group(Cg, negA, negB, g, beta, C):
        Cg = np.ascontiguousarray(Cg, np.int32); M, N = Cg.shape
        negA = np.ascontiguousarray(negA, np.int32); negB = np.ascontiguousarray(negB, np.int32)
        C = np.ascontiguousarray(C, np.float64).copy()
        _oo.oo_reconstruct1_group(_p(Cg), _p(negA), _p(negB), M, N, g, beta, _p(C))
        return C

    @staticmethod
    def _pipeline(fn, A, B, S):
        A = _f64(A); B = _f64(B)
        M, K = A.shape; N = B.shape[1]
        C = np.empty((M, N), np.float64)
        sA = np.empty(M, np.int32); sB = np.empty(N, np.int32)
        As = np.empty((S, M, K), np.int8); Bs = np.empty((S, K, N), np.int8)
        Ct = np.empty((S, M, N), np.int32)
        rc = fn(_p(A), _p(B), M, N, K, S, _p(C), _p(sA), _p(sB), _p(As), _p(Bs), _p(Ct))
        if rc != 0:
            raise ValueError(f"oracle rejected S={S}")
        return dict(C=C, shift_A=sA, shift_B=sB, A_slices=As, B_slices=Bs, C_tc=Ct)

    @classmethod
    def scheme2(cls, A, B, S):
        """Whole Scheme II pipeline; returns C and every intermediate."""
        return cls._pipeline(_oo.oo_scheme2_gemm, A, B, S)

    @classmethod
    def scheme1(cls, A, B, S):
        """Whole Scheme I pipeline; C_tc plane g-2 holds group g."""
        return cls._pipeline(_oo.oo_scheme1_gemm, A, B, S)

    @staticmethod
    def gemm_fp128(A, B):
        A = _f64(A); B = _f64(B); M, K = A.shape; N = B.shape[1]
        C = np.empty((M, N), np.float64)
        _oo.oo_gemm_fp128(_p(A), _p(B), M, N, K, _p(C))
        return C

    @staticmethod
    def gemm_fp128_sampled(A, B, ii, jj):
        A = _f64(A); B = _f64(B); M, K = A.shape; N = B.shape[1]
        ii = np.ascontiguousarray(ii, np.int64); jj = np.ascontiguousarray(jj, np.int64)
        out = np.empty(len(ii), np.float64)
        _oo.oo_gemm_fp128_sampled(_p(A), _p(B), M, N, K, _p(ii), _p(jj), len(ii), _p(out))
        return out

    @staticmethod
    def gemm_dd(A, B):
        A = _f64(A); B = _f64(B); M, K = A.shape; N = B.shape[1]
        C = np.empty((M, N), np.float64)
        _oo.oo_gemm_dd(_p(A), _p(B), M, N, K, _p(C))
        return C

    @staticmethod
    def num_threads():
        return int(_oo.oo_num_threads())


# ------------------------------------------------------------------ the reference's own kernels
class Ref:
    """The reference's kernel source run on the host (oracle/_ref/libozaref_cpu.so)."""

    @staticmethod
    def generate_matrix(rows, cols, phi=0.5, seed=42):
        """The reference's seeded generator (utils/matrix_gen.hpp:15-34)."""
        out = np.empty((rows, cols), np.float64)
        _ref.ref_generate_matrix(int(rows), int(cols), float(phi), int(seed), _p(out))
        return out

    @staticmethod
    def tables():
        mod = np.zeros(MAX_SLICES, np.uint8)
        M = np.zeros((MAX_SLICES, 4), np.uint64); Mh = np.zeros((MAX_SLICES, 4), np.uint64)
        P = np.zeros((MAX_SLICES, MAX_SLICES, 4), np.uint64); I = np.zeros((MAX_SLICES, MAX_SLICES), np.uint64)
        _ref.ref_get_tables(_p(mod), _p(M), _p(Mh), _p(P), _p(I))
        return mod, M, Mh, P, I

    @staticmethod
    def beta(K):
        return int(_ref.ref_scheme1_beta(K))

    @staticmethod
    def k_param(S, K):
        return int(_ref.ref_scheme2_kparam(S, K))

    @staticmethod
    def row_shifts(A, offset):
        A = _f64(A); out = np.empty(A.shape[0], np.int32)
        _ref.ref_row_shifts(_p(A), A.shape[0], A.shape[1], offset, _p(out))
        return out

    @staticmethod
    def col_shifts(B, offset):
        B = _f64(B); out = np.empty(B.shape[1], np.int32)
        _ref.ref_col_shifts(_p(B), B.shape[0], B.shape[1], offset, _p(out))
        return out

    @staticmethod
    def slice2(X, shifts, per_row, S):
        X = _f64(X); sh = np.ascontiguousarray(shifts, np.int32)
        out = np.empty((S,) + X.shape, np.int8)
        _ref.ref_slice2(_p(X), X.shape[0], X.shape[1], _p(sh), int(per_row), S, _p(out))
        return out

    @staticmethod
    def slice1(X, neg_exp, per_row, S, beta):
        X = _f64(X); sh = np.ascontiguousarray(neg_exp, np.int32)
        out = np.empty((S,) + X.shape, np.int8)
        _ref.ref_slice1(_p(X), X.shape[0], X.shape[1], _p(sh), int(per_row), S, beta, _p(out))
        return out

    @staticmethod
    def reconstruct2(Ctc, sA, sB):
        Ctc = np.ascontiguousarray(Ctc, np.int32); S, M, N = Ctc.shape
        C = np.empty((M, N), np.float64)
        _ref.ref_reconstruct2(_p(Ctc), _p(np.ascontiguousarray(sA, np.int32)),
                              _p(np.ascontiguousarray(sB, np.int32)), M, N, S, _p(C))
        return C

    @staticmethod
    def reconstruct1_group(Cg, negA, negB, g, beta, C):
        Cg = np.ascontiguousarray(Cg, np.int32); M, N = Cg.shape
        C = np.ascontiguousarray(C, np.float64).copy()
        _ref.ref_reconstruct1_group(_p(Cg), _p(np.ascontiguousarray(negA, np.int32)),
                                    _p(np.ascontiguousarray(negB, np.int32)), M, N, g, beta, _p(C))
        return C

    @staticmethod
    def cpu_pipeline(scheme, A, B, S, scratch=None):
        """The reference's whole pipeline on the host (steps 1/2/4 are its own
        kernels; step 3 is an exact CPU INT8 GEMM).  `scratch` reuses buffers."""
        A = _f64(A); B = _f64(B); M, K = A.shape; N = B.shape[1]
        if scratch is None:
            scratch = dict(C=np.empty((M, N)), sA=np.empty(M, np.int32), sB=np.empty(N, np.int32),
                           As=np.empty(S * M * K, np.int8), Bs=np.empty(S * K * N, np.int8),
                           Ct=np.empty((S if scheme == 2 else 1) * M * N, np.int32),
                           Bt=np.empty(K * N, np.int8))
        s = scratch
        fn = _ref.ref_cpu_scheme2_gemm if scheme == 2 else _ref.ref_cpu_scheme1_gemm
        fn(_p(A), _p(B), _p(s["C"]), M, N, K, S, _p(s["sA"]), _p(s["sB"]), _p(s["As"]), _p(s["Bs"]),
           _p(s["Ct"]), _p(s["Bt"]))
        return s["C"], scratch


# ------------------------------------------------------------------ error metrics
def error_metrics(expected, actual):
    """Max abs / max relative / Frobenius errors, relative error falling back to
    the absolute one where the expected value is 0 (utils/matrix_compare.hpp:24-65)."""
    e = np.asarray(expected, np.float64).ravel(); a = np.asarray(actual, np.float64).ravel()
    d = a - e
    ad = np.abs(d)
    ae = np.abs(e)
    rel = np.where(ae > 0, ad / np.where(ae > 0, ae, 1.0), ad)
    fe = float(np.sqrt(np.sum(d * d)))
    fx = float(np.sqrt(np.sum(e * e)))
    return dict(max_abs=float(ad.max(initial=0.0)), max_rel=float(rel.max(initial=0.0)), frobenius=fe,
                rel_frobenius=fe / fx if fx > 0 else fe)
