"""Runs one engine workload a few times, for profilers (ncu) and quick timing.

    python -m fft_b200.prof rfft2 --prec f64 --batch 16 --reps 3
    python -m fft_b200.prof roundtrip --prec f64 --batch 32 --reps 5 --pipe off
    python -m fft_b200.prof c2c --n 1024 --prec f64 --batch 4096 --reps 3
    python -m fft_b200.prof fftn --shape 256,256,256 --prec f32mixed
    python -m fft_b200.prof rfft2 --prec f64 --wisdom wisdom.json
    python -m fft_b200.prof uneven-classes --prec f32mixed
    python -m fft_b200.prof spectrogram --prec f32mixed --n 4194304
    python -m fft_b200.prof filter2 --prec f32mixed --shape 512,512 --batch 32

Prints the CUDA-event time per repetition (taken without a profiler; under a
profiler the printed times are not measurements).  `roundtrip` is RFFT2 then
IRFFT2 (the bench step).  `uneven-classes` times the length classes of the
uneven batch (4096 complex64 signals, lengths drawn from seed 2 over
{60, 128, 360, 1000, 1009, 4096, 10007, 65536}) one class at a time.
`spectrogram` is the fused spectrogram of an --n-sample signal (Hann 2048,
overlap 1536); `filter2` the 2-D spectral filter forward then backward.
`--pipe off` turns the TMA-fed persistent line kernel off for comparison;
`--pdl` sets the programmatic dependent-launch mode of the line kernels.
"""
import argparse

import numpy as np
import torch

from .device import DevicePlan


def _time(run, reps):
    run()
    torch.cuda.synchronize()
    out = []
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        run()
        e1.record()
        torch.cuda.synchronize()
        out.append(e0.elapsed_time(e1))
    return out


def uneven_classes(prec, reps):
    g = np.random.default_rng(2)
    lens = [int(v) for v in g.choice([60, 128, 360, 1000, 1009, 4096, 10007, 65536], 4096)]
    cdt = torch.complex128 if prec == "f64" else torch.complex64
    tot = 0.0
    for n in sorted(set(lens)):
        b = lens.count(n)
        p = DevicePlan("c2c", prec, [n], batch=b)
        x = torch.randn(b, n, dtype=cdt, device="cuda")
        y = torch.empty_like(x)
        ms = min(_time(lambda: p.c2c(x, out=y), reps))
        tot += ms
        eng = [a.get("engine") for a in p.describe().get("axes", [])]
        print("n=%6d signals=%4d points=%9d  %.4f ms  %7.1f GB/s  engine=%s"
              % (n, b, n * b, ms, n * b * 2 * x.element_size() / ms / 1e6, eng), flush=True)
    print("sum of classes %.4f ms, points %d" % (tot, sum(lens)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["rfft2", "irfft2", "roundtrip", "c2c", "fftn", "r2c", "uneven-classes",
                                     "spectrogram", "filter2"])
    ap.add_argument("--prec", default="f64")
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--shape", default="1024,1024")
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--wisdom", default=None, help="tuning settings (JSON) to import first")
    ap.add_argument("--pipe", default="on", choices=["on", "off"], help="TMA-fed persistent line kernel")
    ap.add_argument("--lanes", type=int, default=0, help="lanes of blocked plans (0: default)")
    ap.add_argument("--sched", default="", help="schedule variants, e.g. 1024:1,512:1")
    ap.add_argument("--pdl", type=int, default=-1, help="dependent-launch mode 0/1/2 (-1: the default)")
    a = ap.parse_args()
    torch.cuda.set_device(0)
    from . import tune
    tune.set_tma_pipeline(a.pipe == "on")
    tune.set_lanes(a.lanes)
    if a.pdl >= 0:
        tune.set_dependent_launch(a.pdl)
    if a.wisdom:
        with open(a.wisdom) as f:
            tune.import_wisdom(f.read())
    if a.sched:
        from ._lib import check, lib
        from .device import PRECISIONS
        for item in a.sched.split(","):
            n, v = item.split(":")
            check(lib().gofft_set_schedule(PRECISIONS[a.prec], int(n), int(v)))
    if a.case == "uneven-classes":
        uneven_classes(a.prec, a.reps)
        return
    g = np.random.default_rng(0)
    rdt = torch.float64 if a.prec == "f64" else torch.float32
    cdt = torch.complex128 if a.prec == "f64" else torch.complex64
    shape = [int(s) for s in a.shape.split(",")]
    if a.case == "spectrogram":
        from .device import spectrogram, window
        sig = torch.from_numpy(g.standard_normal(a.n)).to(rdt).cuda()
        win = window("hann", 2048, a.prec)

        def run():
            spectrogram(sig, 2048, 1536, win, 1.0, a.prec)
    elif a.case == "filter2":
        from .function import SpectralFilter2
        f = SpectralFilter2(a.prec, shape[0], shape[1], batch=a.batch)
        xf = torch.from_numpy(g.random((a.batch, shape[0] * shape[1]))).to(rdt).cuda()
        K = shape[1] // 2 + 1
        Hf = torch.from_numpy(g.standard_normal(shape[0] * K) + 1j * g.standard_normal(shape[0] * K)).to(cdt).cuda()
        yf = f.Forward(xf, Hf)

        def run():
            f.plan.filter2(xf, Hf, out=yf, saved=f.saved)
            f.plan.vjp_filter2(yf, Hf, saved=f.saved, scratch=f.saved)
    elif a.case in ("rfft2", "irfft2", "r2c", "roundtrip"):
        if a.case == "r2c":
            shape = [a.n]
        p = DevicePlan("r2c", a.prec, shape, batch=a.batch)
        x = torch.from_numpy(g.standard_normal((a.batch, int(np.prod(shape))))).to(rdt).cuda()
        X = p.r2c(x)
        back = torch.empty_like(x)

        def run():
            if a.case == "irfft2":
                p.c2r(X, out=back)
            elif a.case == "roundtrip":
                p.r2c(x, out=X)
                p.c2r(X, out=back)
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
    for ms in _time(run, a.reps):
        print("%s %s pipe=%s %.4f ms" % (a.case, a.prec, a.pipe, ms))
    tune.pipeline_status()


if __name__ == "__main__":
    main()
