"""Micro-benchmark of the tensor-core 3x3x3 convolutions (forward and weight gradient) on one
channels-last BF16 volume.

    python -m waveletpotentials_b200.conv_bench [--n 64] [--c 32] [--reps 10] [--profile-region]

Prints one line per kernel with its CUDA-event time and TFLOP/s (2 * 27 * c * c * n^3 flops).
"""
from __future__ import annotations

import argparse

import torch

from . import api


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--c", type=int, default=32)
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--profile-region", action="store_true")
    a = ap.parse_args()
    n, c = a.n, a.c
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn((n, n, n, c), device="cuda", generator=g).to(torch.bfloat16)
    w = (torch.randn((27, c, c), device="cuda", generator=g) * 0.05).to(torch.bfloat16)
    out = torch.empty_like(x)
    dw = torch.zeros((27, c, c), device="cuda")
    for _ in range(3):
        api.conv3_forward(out, x, w)
        api.conv3_wgrad(dw, x, out)
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    if a.profile_region:
        torch.cuda.profiler.start()
    ev[0].record(st)
    for _ in range(a.reps):
        api.conv3_forward(out, x, w)
    ev[1].record(st)
    for _ in range(a.reps):
        api.conv3_wgrad(dw, x, out)
    ev[2].record(st)
    torch.cuda.synchronize()
    if a.profile_region:
        torch.cuda.profiler.stop()
    fl = 2.0 * 27 * c * c * n ** 3
    for name, t in (("conv3_forward", ev[0].elapsed_time(ev[1]) / a.reps),
                    ("conv3_wgrad", ev[1].elapsed_time(ev[2]) / a.reps)):
        print(f"{name} n={n} c={c}: {t:.4f} ms, {fl / t / 1e9:.1f} TFLOP/s")


if __name__ == "__main__":
    main()
