"""Throughput of the split-precision batched ZGEMM against cuBLAS ZGEMM.

    python -m tups_b200.split_bench [--Nz 576] [--batch 64] [--slices 2 3 4 5 6 7 8] [--reps 5]

Batched C_b = A_b B_b with M = N = Nz and K = 2 Nz, the shape of the BSE
GEMM [Gamma chi | F] [F ; chi Gamma] for Nz = Nl * Nf.  Random complex128
inputs (seeded), device-resident; CUDA-event timing on the launching stream
after one untimed call.  One JSON line per slice count with the effective
FP64-equivalent TFLOP/s (8 M N K per batch entry), the int8 tensor rate and
the relative error against the FP64 product of the first batch entry.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json


def run(Nz: int, batch: int, slices, reps: int = 5, device: int = 0, check: bool = True):
    import torch
    from . import load
    lib = load()
    torch.cuda.set_device(device)
    M = N = Nz
    K = 2 * Nz
    g = torch.Generator(device="cuda")
    g.manual_seed(1234)
    # column-major per batch entry = transposed row-major
    A = torch.randn((batch, K, M), dtype=torch.complex128, device="cuda", generator=g)
    B = torch.randn((batch, N, K), dtype=torch.complex128, device="cuda", generator=g)
    Cm = torch.zeros((batch, N, M), dtype=torch.complex128, device="cuda")
    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    At, Bt = A.transpose(1, 2), B.transpose(1, 2)
    ref = torch.matmul(At, Bt)

    def time_cublas() -> float:
        for _ in range(3):
            torch.matmul(At, Bt)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            torch.matmul(At, Bt)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    zgemm_ms = time_cublas()
    flops = 8.0 * M * N * K * batch
    out = []
    for s in slices:
        ws = lib.tups_zgemm_split_workspace(batch, M, N, K, s)
        work = torch.empty(ws, dtype=torch.uint8, device="cuda")
        args = (batch, M, N, K, C.c_void_p(A.data_ptr()), C.c_void_p(B.data_ptr()), C.c_void_p(Cm.data_ptr()), s,
                C.c_void_p(work.data_ptr()), ws, C.c_void_p(stream.cuda_stream))
        rc = lib.tups_zgemm_split(*args)
        if rc:
            raise RuntimeError(f"tups_zgemm_split failed with {rc}")
        err = None
        if check:
            got = Cm[0].transpose(0, 1)
            err = float((got - ref[0]).abs().max() / ref[0].abs().max())
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            lib.tups_zgemm_split(*args)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        pairs = s * (s + 1) // 2
        line = {"Nz": Nz, "batch": batch, "slices": s, "ms": ms, "effective_tflops": flops / ms / 1e9,
                "int8_tops": 2.0 * pairs * M * (2 * N) * (2 * K) * batch / ms / 1e9,
                "cublas_zgemm_ms": zgemm_ms, "cublas_zgemm_tflops": flops / zgemm_ms / 1e9,
                "speedup_vs_cublas": zgemm_ms / ms, "rel_err_vs_fp64": err}
        out.append(line)
        del work
    # cuBLAS again after the split runs; keep its faster time
    z2 = time_cublas()
    if z2 < zgemm_ms:
        for line in out:
            line["cublas_zgemm_ms"] = z2
            line["cublas_zgemm_tflops"] = flops / z2 / 1e9
            line["speedup_vs_cublas"] = z2 / line["ms"]
    return out


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--Nz", type=int, default=576)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--slices", type=int, nargs="+", default=[2, 3, 4, 5, 6, 7, 8])
    ap.add_argument("--reps", type=int, default=5)
    a = ap.parse_args(argv)
    lines = run(a.Nz, a.batch, a.slices, a.reps)
    for line in lines:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
