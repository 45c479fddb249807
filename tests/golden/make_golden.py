#!/usr/bin/env python3
"""Generates the committed golden fixtures in tests/golden/ from the reference
itself (IlyaNyrkov/ozablas), so the tests can pin parity on machines where
the reference tree is absent.

  * generator.npz  -- first values of the reference's matrix generator
    (utils/matrix_gen.hpp) for a few (rows, cols, phi, seed), produced by a
    tiny C++ program compiled here against that header.
  * crt_tables.npz -- the reference's CRT tables (src/common/crt_tables.hpp),
    read through oracle/_ref/libozaref_cpu.so.
  * pipeline_*.npz -- inputs, shifts, slices/residues, INT32 products and C of
    the reference's own step-1/2/4 kernels (run on the host by the shim) with
    an exact INT8 GEMM for step 3, for Scheme II and Scheme I cases including
    exponent edge cases.

Usage: python tests/golden/make_golden.py [--ref PATH]
(PATH: a checkout of the reference tree; default $OZABLAS_REF, else a
directory named "reference" beside this repository).
"""
import argparse
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

GEN_CASES = [(4, 5, 0.5, 42), (3, 7, 2.0, 43), (2, 9, 4.0, 7), (1, 16, 0.0, 1234)]


def generator_fixture(ref):
    src = r'''
#include <cstdio>
#include <cstdlib>
#include "matrix_gen.hpp"
int main(int argc, char** argv) {
    int r = atoi(argv[1]), c = atoi(argv[2]); double phi = atof(argv[3]); int seed = atoi(argv[4]);
    auto m = matrix_utils::generation::generate_ozaki_matrix<double>(r, c, phi, seed);
    for (double v : m) printf("%a\n", v);
    return 0;
}
'''
    with tempfile.TemporaryDirectory() as td:
        cpp = os.path.join(td, "gen.cpp")
        exe = os.path.join(td, "gen")
        with open(cpp, "w") as f:
            f.write(src)
        subprocess.run(["/usr/bin/g++", "-O2", "-std=c++17", f"-I{ref}/utils", cpp, "-o", exe], check=True)
        out = {}
        for i, (r, c, phi, seed) in enumerate(GEN_CASES):
            txt = subprocess.run([exe, str(r), str(c), repr(phi), str(seed)], check=True, capture_output=True,
                                 text=True).stdout.split()
            out[f"case{i}"] = np.array([float.fromhex(t) for t in txt]).reshape(r, c)
            out[f"params{i}"] = np.array([r, c, phi, seed], dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, "generator.npz"), **out)


def edge_matrices(M, N, K, seed, tiny=True):
    """Exponent edge cases.  `tiny` adds a row of subnormals whose maximum lies
    below 2^-1024; Scheme I fixtures leave it out because the reference then
    casts +-inf to int8 (0 * inf = NaN for zeros, inf otherwise), which is
    undefined in C++ and differs between the host-compiled kernel (0) and the
    GPU build (saturation); the GPU tests pin that case against the GPU build."""
    import ozablas_b200 as oz
    A = oz.generate_matrix(M, K, 4.0, seed)
    B = oz.generate_matrix(K, N, 4.0, seed + 1)
    rng = np.random.default_rng(seed)
    A[rng.random(A.shape) < 0.05] = 0.0
    B[rng.random(B.shape) < 0.05] = 0.0
    A[2, :] = 0.0
    B[:, 3] = 0.0
    A[1, :] *= 2.0 ** 300
    A[4, :] *= 2.0 ** -300
    B[:, 5] *= 2.0 ** 300
    B[:, 6] *= 2.0 ** -300
    A[7, :] = np.ldexp(1.0, np.arange(K) % 9 - 4)
    A[8, :] = np.nextafter(np.ldexp(1.0, np.arange(K) % 5), 0.0)
    if tiny:
        A[9, :] = 5e-324 * (np.arange(K) + 1)
    B[:, 10] = -2.2250738585072014e-308 * (np.arange(K) + 1)
    return A, B


def pipeline_fixture(name, A, B, scheme, S):
    from oracle import Oracle, Ref
    M, K = A.shape
    N = B.shape[1]
    out = dict(A=A, B=B, scheme=np.int32(scheme), S=np.int32(S))
    if scheme == 2:
        kp = Ref.k_param(S, K)
        sA, sB = Ref.row_shifts(A, kp), Ref.col_shifts(B, kp)
        As, Bs = Ref.slice2(A, sA, 1, S), Ref.slice2(B, sB, 0, S)
        Ct = np.stack([Oracle.gemm_i8(As[s], Bs[s]) for s in range(S)])
        C = Ref.reconstruct2(Ct, sA, sB)
        out.update(k_param=np.int32(kp))
    else:
        beta = Ref.beta(K)
        sA, sB = Ref.row_shifts(A, 0), Ref.col_shifts(B, 0)
        As, Bs = Ref.slice1(A, sA, 1, S, beta), Ref.slice1(B, sB, 0, S, beta)
        C = np.zeros((M, N))
        Ct = np.zeros((S, M, N), np.int32)
        for g in range(2, S + 2):
            acc = None
            for s in range(1, g):
                t = g - s
                if s > S or t > S:
                    continue
                acc = Oracle.gemm_i8(As[s - 1], Bs[t - 1], acc)
            Ct[g - 2] = acc
            C = Ref.reconstruct1_group(acc, sA, sB, g, beta, C)
        out.update(beta=np.int32(beta))
    out.update(shift_A=sA, shift_B=sB, A_slices=As, B_slices=Bs, C_tc=Ct, C=C)
    np.savez_compressed(os.path.join(HERE, f"pipeline_{name}.npz"), **out)


def main():
    ap = argparse.ArgumentParser()
    default_ref = os.environ.get("OZABLAS_REF") or os.path.join(os.path.dirname(ROOT), "reference")
    ap.add_argument("--ref", default=default_ref)
    args = ap.parse_args()
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), f"REF={args.ref}"], check=True)
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "ozablas_b200", "csrc")], check=True)
    from oracle import Ref
    generator_fixture(args.ref)
    mod, M, Mh, P, I = Ref.tables()
    np.savez_compressed(os.path.join(HERE, "crt_tables.npz"), moduli=mod, M=M, M_half=Mh, partial=P, inv=I)
    import ozablas_b200 as oz
    A = oz.generate_matrix(48, 64, 0.5, 42)
    B = oz.generate_matrix(64, 40, 0.5, 43)
    for S in (1, 7, 8, 16, 20):
        pipeline_fixture(f"s2_seeded_S{S}", A, B, 2, S)
    for S in (1, 4, 8):
        pipeline_fixture(f"s1_seeded_S{S}", A, B, 1, S)
    Ae, Be = edge_matrices(24, 20, 40, 5)
    for S in (8, 19):
        pipeline_fixture(f"s2_edge_S{S}", Ae, Be, 2, S)
    Ae, Be = edge_matrices(24, 20, 40, 5, tiny=False)
    pipeline_fixture("s1_edge_S7", Ae, Be, 1, 7)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
