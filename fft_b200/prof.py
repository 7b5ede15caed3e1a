"""Runs one engine workload a few times, for profilers (ncu) and quick timing.

    python -m fft_b200.prof rfft2 --prec f64 --batch 16 --reps 3
    python -m fft_b200.prof c2c --n 1024 --prec f64 --batch 4096 --reps 3
    python -m fft_b200.prof fftn --shape 256,256,256 --prec f32mixed
    python -m fft_b200.prof rfft2 --prec f64 --wisdom wisdom.json

Prints the CUDA-event time per repetition (taken without a profiler; under a
profiler the printed times are not measurements).
"""
import argparse

import numpy as np
import torch

from .device import DevicePlan


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["rfft2", "irfft2", "c2c", "fftn", "r2c"])
    ap.add_argument("--prec", default="f64")
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--shape", default="1024,1024")
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--wisdom", default=None, help="tuning settings (JSON) to import first")
    a = ap.parse_args()
    torch.cuda.set_device(0)
    if a.wisdom:
        from .tune import import_wisdom
        with open(a.wisdom) as f:
            import_wisdom(f.read())
    g = np.random.default_rng(0)
    rdt = torch.float64 if a.prec == "f64" else torch.float32
    cdt = torch.complex128 if a.prec == "f64" else torch.complex64
    shape = [int(s) for s in a.shape.split(",")]
    if a.case in ("rfft2", "irfft2", "r2c"):
        if a.case == "r2c":
            shape = [a.n]
        p = DevicePlan("r2c", a.prec, shape, batch=a.batch)
        x = torch.from_numpy(g.standard_normal((a.batch, int(np.prod(shape))))).to(rdt).cuda()
        X = p.r2c(x)

        def run():
            if a.case == "irfft2":
                p.c2r(X)
            else:
                p.r2c(x, out=X)
    else:
        if a.case == "c2c":
            shape = [a.n]
        p = DevicePlan("c2c", a.prec, shape, batch=a.batch)
        n = int(np.prod(shape))
        x = torch.from_numpy(g.standard_normal((a.batch, n)) + 1j * g.standard_normal((a.batch, n))).to(cdt).cuda()
        y = torch.empty_like(x)

        def run():
            p.c2c(x, out=y)
    run()
    torch.cuda.synchronize()
    for _ in range(a.reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        run()
        e1.record()
        torch.cuda.synchronize()
        print("%s %s %.3f ms" % (a.case, a.prec, e0.elapsed_time(e1)))


if __name__ == "__main__":
    main()
