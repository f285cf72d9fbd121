"""Times the tensor-core GEMM (oems_tc_gemm_bf16) on one shape.

    python -m openems_b200.gemm_bench M N K [--calls 3] [--time 50]

Random bf16 A [M, K] and B [N, K] on the device; `--calls` calls of
oems_tc_gemm_bf16 (C = A B^T, f32), then the relative error against
torch's float product; with --time R, R more calls between CUDA events
(the host's tensor-map encoding included) and the TFLOP/s.  Prints one JSON
line.
"""
from __future__ import annotations

import argparse
import json


def main(argv=None):
    import torch

    from . import _native as N
    p = argparse.ArgumentParser()
    p.add_argument("M", type=int)
    p.add_argument("N", type=int)
    p.add_argument("K", type=int)
    p.add_argument("--calls", type=int, default=3)
    p.add_argument("--time", type=int, default=0)
    a = p.parse_args(argv)
    g = torch.Generator(device="cpu").manual_seed(1)
    A = torch.randn(a.M, a.K, generator=g).to(torch.bfloat16).cuda()
    B = torch.randn(a.N, a.K, generator=g).to(torch.bfloat16).cuda()
    C = torch.zeros(a.M, a.N, device="cuda")
    lib = N.lib()
    stream = torch.cuda.current_stream().cuda_stream

    def call():
        N.check(lib.oems_tc_gemm_bf16(A.data_ptr(), a.K, B.data_ptr(), a.K, C.data_ptr(), a.N, a.M, a.N, a.K,
                                      0.0, None, stream))

    for _ in range(a.calls):
        call()
    torch.cuda.synchronize()
    N.check(lib.oems_tc_check(None))
    ref = A.float() @ B.float().T
    out = {"M": a.M, "N": a.N, "K": a.K, "rel_err": ((C - ref).abs().max() / ref.abs().max()).item()}
    if a.time > 0:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.time):
            call()
        e1.record()
        torch.cuda.synchronize()
        N.check(lib.oems_tc_check(None))
        ms = e0.elapsed_time(e1) / a.time
        out.update({"ms": ms, "tflops": 2.0 * a.M * a.N * a.K / (ms * 1e-3) / 1e12})
    print(json.dumps(out))


if __name__ == "__main__":
    main()
