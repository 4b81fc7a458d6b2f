#!/usr/bin/env python
"""Benchmark of the B200 CBPDN ADMM solvers (ADMM iterations per second).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config C] [--impl ours|reference]

Workload (default --config 4, the largest single-GPU configuration): one
2048x2048 float32 image, 256 unit-norm 16x16 Gaussian filters, S synthesised
from Bernoulli(0.01) x N(0,1) sparse maps plus N(0, 0.01^2) noise and
mean-subtracted (seeded); a step is one cbpdn solve (lambda 0.02, AutoRho on)
of 100 ADMM iterations (no early stop).  Configs 0 (256x256, M=64, fixed rho),
1 (cbpdngrd + cbpdnmsk at 512x512, M=100), 2 (batched, 64 uneven images) and
3 (forward + adjoint of 200 unrolled iterations) are selectable.  Data are
synthetic, drawn on the host (torch CPU generator, float64 FFTs) so that both
arms see the same problem.

Printed JSON line (rank 0): ``value`` = ADMM iterations per second with inputs
resident in device memory, summed over ranks (each rank runs an independent
replica: the path has no data-path collective); ``e2e`` = the same metric
through the reference-facing API (numpy host buffers in and out, host<->device
copies inside the timed region); ``roofline`` = algorithmic HBM bytes of one
ADMM iteration (4R + 6C + 2C_D, R = 4 M H W, C = C_D = 8 M H (W/2+1)) over the
measured device time of one iteration (CUDA events around every kernel of the
timed solves), against the measured HBM copy bandwidth; ``cpu_baseline`` = the
FP64 CPU restatement of the algorithm timed on this host on a bounded sample
(the first n iterations); ``rel_err`` = the GPU solver's coefficient maps and
functional after those n iterations against that FP64 run.

``--impl reference`` times the reference algorithm's CPU implementation (the
FP64 restatement with every host thread; the reference ships no CPU solver of
its own) on the same workload: each step continues one solve by a bounded
number of iterations.  It loads nothing of this package.
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "sporco-cuda_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

F32 = np.float32

METRIC = ("ADMM iters/s & HBM GB/s (plain vs batched vs fwd+adjoint), "
          "rel err ≤1e-4 vs FP64")

CONFIGS = {
    0: dict(workload="cbpdn 256x256 M=64 8x8, 200 iterations, fixed rho",
            H=256, W=256, M=64, K=8, density=0.01, lmbda=0.05, mu=0.0,
            variants=["cbpdn"], iters=200, autorho=False, mask_p=None, check_iters=40),
    1: dict(workload="cbpdngrd + cbpdnmsk 512x512 M=100 12x12, 500 iterations, AutoRho",
            H=512, W=512, M=100, K=12, density=0.005, lmbda=0.05, mu=0.1,
            variants=["cbpdngrd", "cbpdnmsk"], iters=500, autorho=True, mask_p=0.7,
            check_iters=20),
    4: dict(workload="cbpdn 2048x2048 M=256 16x16, 100 iterations, AutoRho",
            H=2048, W=2048, M=256, K=16, density=0.01, lmbda=0.02, mu=0.0,
            variants=["cbpdn"], iters=100, autorho=True, mask_p=None, check_iters=2),
    2: dict(workload="batched cbpdnmsk: 64 images, sides from {128..1024} (H, W independent), "
                     "M=64 12x12, per-image masks and lambda, AutoRho, RelStopTol 1e-4, cap 1000",
            H=None, W=None, M=64, K=12, density=0.005, lmbda=None, mu=0.0,
            variants=["cbpdnmsk"], iters=1000, autorho=True, mask_p=None, nimg=64,
            sides=(128, 192, 256, 384, 512, 768, 1024)),
    3: dict(workload="differentiable cbpdn: 16 images 256x256, M=32 11x11, 200 unrolled "
                     "iterations, loss ||D*X - S_clean||^2 + 0.01||X||_1, backward to D and S",
            H=256, W=256, M=32, K=11, density=0.01, lmbda=0.05, mu=0.0, nimg=16,
            variants=["cbpdn"], iters=200, autorho=False, mask_p=None),
    # 1024x1024 with the maps of the 2048x2048 problem: the column pass's
    # per-CTA work of that problem at a quarter of its memory (3 GB), for
    # kernel profiles
    10: dict(workload="cbpdn 1024x1024 M=256 16x16, 20 iterations, AutoRho (profiling case)",
             H=1024, W=1024, M=256, K=16, density=0.01, lmbda=0.02, mu=0.0,
             variants=["cbpdn"], iters=20, autorho=True, mask_p=None, check_iters=3),
    # small 2048x2048 case for kernel profiles (2 GB on the device)
    9: dict(workload="cbpdn 2048x2048 M=24 16x16, 20 iterations, AutoRho (profiling case)",
            H=2048, W=2048, M=24, K=16, density=0.01, lmbda=0.02, mu=0.0,
            variants=["cbpdn"], iters=20, autorho=True, mask_p=None, check_iters=5),
}
DEFAULT_CONFIG = 4


# ---------------------------------------------------------------- helpers --

def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def opt_for(cfg, variant, iters=None):
    lam = np.float32(cfg["lmbda"])
    opt = {"Verbose": False, "MaxMainIter": iters or cfg["iters"], "RelStopTol": 0.0,
           "AbsStopTol": 0.0,
           "RelaxParam": 1.8, "L1Weight": 1.0, "GradWeight": 1.0,
           "AutoRho": {"Enabled": cfg["autorho"], "Period": 1, "Scaling": 1000.0,
                       "RsdlRatio": 1.2, "RsdlTarget": None, "AutoScaling": True,
                       "StdResiduals": False}}
    opt["rho"] = None if cfg["autorho"] else float(np.float32(50 * lam + 1))
    return opt


# Column lengths with compiled transform plans (the convolution column solve
# needs one for its per-tile transforms).
SPEC_COL = {16, 32, 64, 128, 256, 512, 1024, 2048, 48, 96, 192, 384, 768, 1536}
SMEM_MAX = 227 * 1024  # shared memory of one CTA


def graded_bytes(H, W, M, images=1):
    """Algorithmic HBM bytes of one ADMM iteration of `images` images of one
    size (the graded byte model).  R = 4 M H W, C = 8 M H (W/2+1); p = 1 when
    one map's half-spectrum fits in one CTA's shared memory (the 2-D FFT can
    stay on chip), else 2.  Per image 4R + 6C (p = 2) or 4R + 2C (p = 1): Y
    and U read and written once, three (or one) spectrum round trips; per
    size the dictionary spectra are read twice (p = 2) or once (p = 1)."""
    R = 4.0 * M * H * W
    Cs = 8.0 * M * H * (W // 2 + 1)
    p = 1 if 8 * H * (W // 2 + 1) <= SMEM_MAX else 2
    return images * (4 * R + (6 if p == 2 else 2) * Cs) + (2 if p == 2 else 1) * Cs


def graded_kernel_bytes(H, W, M):
    """The graded bytes of one image's iteration split by pass: the row pass
    reads and writes Y, U and the spectra (4R + 2C); the column pass takes
    the remaining spectrum round trips and the dictionary reads (4C + 2C_D
    when p = 2, C_D when p = 1)."""
    R = 4.0 * M * H * W
    Cs = 8.0 * M * H * (W // 2 + 1)
    p = 1 if 8 * H * (W // 2 + 1) <= SMEM_MAX else 2
    return {"row_kernel": 4 * R + 2 * Cs, "col_kernel": (6 * Cs) if p == 2 else Cs}


# DRAM bytes per launch and map measured by ncu (dram__bytes_read.sum +
# dram__bytes_write.sum, one-kernel captures) for kernels whose traffic grows
# in proportion to the maps, with the capture each comes from (kernels as of
# the commit named there).
MEASURED_TRAFFIC_PER_MAP = {
    (2048, 2048): {"row_kernel": ((807.2e6 + 744.6e6) / 24,
                                  "ncu capture at 2048x2048, M=24 (kernels of commit 193bd5b), "
                                  "scaled by the maps"),
                   "col_kernel": ((454.6e6 + 357.5e6) / 24,
                                  "ncu capture at 2048x2048, M=24 (kernels of commit 193bd5b), "
                                  "scaled by the maps")},
    (512, 512): {"col_kernel": (((216.1e6 + 49.3e6) + (218.5e6 + 56.2e6)) / 2 / 100,
                                "ncu captures at 512x512, M=100, mean of the gradient and "
                                "masked column solves (kernels of commit 2d8664f)")},
}


def design_bytes(H, W, M, variant="cbpdn", K=None):
    """Per-iteration HBM bytes this design moves for one image.  Row pass:
    reads and writes the spectra F (2C) and the state V = Y + U (2R).  Column pass, by
    solve: the plain convolution solves (filters of at most 16 rows,
    compiled column length) read F once and write the correction to it
    (2C; the row pass adds Y - U itself; masked problems read F twice and
    write it whole, 3C); the gradient convolution solve
    (one GradWeight for every map) reads F twice and writes it (3C); the
    transform solve also reads the dictionary spectra twice (+2 C_D,
    C_D = C per image); with a map-dependent gradient term it also writes
    and re-reads the column spectra between its two passes (+2C)."""
    R = 4.0 * M * H * W
    Cs = 8.0 * M * H * (W // 2 + 1)
    grd = variant in ("cbpdngrd", "cbpdngrdmsk")
    per_map = variant == "cbpdngrdmsk"
    conv = not per_map and K is not None and K <= 16 and H in SPEC_COL
    masked = variant in ("cbpdnmsk", "cbpdngrdmsk")
    if conv:
        col = 3 * Cs if grd or masked else 2 * Cs
    else:
        col = 3 * Cs + 2 * Cs + (2 * Cs if grd else 0)
    return 2 * R + 2 * Cs + col


def synth(cfg, seed):
    """Unit-norm Gaussian filters D (M, K, K), S = sum_m d_m * x_m + noise
    (x_m Bernoulli(density) x N(0, 1), drawn as that many uniformly placed
    nonzeros), mean-subtracted, and the Bernoulli observation mask of the
    masked configurations; float32 numpy arrays.  Drawn with the torch CPU
    generator and float64 FFTs on the host, so that every arm of the
    benchmark (including the reference arm, which loads nothing of this
    package) solves the same problem."""
    import torch
    H, W, M, K = cfg["H"], cfg["W"], cfg["M"], cfg["K"]
    g = torch.Generator().manual_seed(seed)
    D = torch.randn((M, K, K), generator=g, dtype=torch.float64)
    D /= torch.sqrt(torch.sum(D * D, dim=(1, 2), keepdim=True))
    Sf = torch.zeros((H, W // 2 + 1), dtype=torch.complex128)
    for m0 in range(0, M, 16):
        m1 = min(M, m0 + 16)
        n = (m1 - m0) * H * W
        nnz = int(round(cfg["density"] * n))
        X0 = torch.zeros(n, dtype=torch.float64)
        X0.index_put_((torch.randint(0, n, (nnz,), generator=g),),
                      torch.randn(nnz, generator=g, dtype=torch.float64), accumulate=True)
        Dp = torch.zeros((m1 - m0, H, W), dtype=torch.float64)
        Dp[:, :K, :K] = D[m0:m1]
        Sf += torch.sum(torch.fft.rfft2(Dp) * torch.fft.rfft2(X0.reshape(m1 - m0, H, W)), dim=0)
    S = torch.fft.irfft2(Sf, s=(H, W)) + 0.01 * torch.randn((H, W), generator=g,
                                                           dtype=torch.float64)
    S = S - S.mean()
    mask = None
    if cfg["mask_p"] is not None:
        mask = (torch.rand((H, W), generator=g, dtype=torch.float64) < cfg["mask_p"]).numpy() \
            .astype(np.float32)
    return D.numpy().astype(np.float32), S.numpy().astype(np.float32), mask


class ClockSampler:
    """nvidia-smi clock / throttle-reason sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def _oracle_args(cfg, variant, D, S, mask, iters):
    """Arguments of the oracle entry point for one variant: D (K, K, M)."""
    Dk = np.ascontiguousarray(np.moveaxis(D, 0, 2))
    opt = opt_for(cfg, variant, iters)
    if variant == "cbpdnmsk":
        return dict(variant=variant, D=Dk, S=S * mask, lmbda=cfg["lmbda"], opt=opt, W=mask)
    return dict(variant=variant, D=Dk, S=S, lmbda=cfg["lmbda"], opt=opt, mu=cfg["mu"])


def cpu_leg(cfg, D, S, mask, iters):
    """The FP64 CPU restatement (map-chunked, torch on every host thread) on
    a bounded sample of the workload: the first `iters` ADMM iterations of
    each variant.  Returns the cpu_baseline record and, per variant, the
    FP64 coefficient maps (H, W, M) and the run's information."""
    import torch
    from oracle import cbpdn_oracle_torch as OT
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    out = {}
    t0 = time.perf_counter()
    for v in cfg["variants"]:
        out[v] = OT.solve(**_oracle_args(cfg, v, D, S, mask, iters))
    dt = time.perf_counter() - t0
    total = iters * len(cfg["variants"])
    rec = {"value": total / dt, "unit": "iter/s", "cores": threads, "kind": "port",
           "sample": "%s: the first %d ADMM iterations of %s from zero (FP64 restatement, "
                     "maps in chunks of 16, torch CPU with %d threads; set-up included)"
                     % (cfg["workload"], iters, " and ".join(cfg["variants"]), threads)}
    return rec, out


# ------------------------------------------------------------------ arms --

def config_dict(cfg, world):
    """The `config` object of the JSON line (the same in both arms)."""
    return {"workload": cfg["workload"], "H": cfg["H"], "W": cfg["W"], "M": cfg["M"],
            "K": cfg["K"], "iterations_per_solve": cfg["iters"],
            "solves_per_step": len(cfg["variants"]),
            "parallelism": "replicas%d" % world if world > 1 else "single",
            "l2": "working set larger than L2 (no flush)" if
            graded_bytes(cfg["H"], cfg["W"], cfg["M"]) > 126e6 else "working set fits in L2"}


def run_ours(args, cfg, rank, world, local_rank):
    import torch
    import sporco_cuda.cbpdn as cb
    from sporco_cuda import _lib, replicas
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    Dh, Sh, maskh = synth(cfg, 12345 + args.config + 1000 * rank)
    D = torch.from_numpy(Dh).to(dev)
    S = torch.from_numpy(Sh).to(dev)
    mask = torch.from_numpy(maskh).to(dev) if maskh is not None else None
    lam = cfg["lmbda"]
    # device-resident solves (one for the timed steps, one with an event pair
    # around every kernel launch for the per-kernel split)
    solves = []
    for v in cfg["variants"]:
        opt = opt_for(cfg, v)
        if v == "cbpdnmsk":
            M1 = cfg["M"] + 1
            Di = torch.zeros((M1, cfg["K"], cfg["K"]), device=dev)
            Di[0, 0, 0] = 1.0
            Di[1:] = D
            l1 = np.ones(M1, np.float32)
            l1[0] = 0.0
            pair = [cb.prepare_device(Di, (S * mask)[None], lam, opt, l1=l1,
                                      mask=mask.to(torch.int32)[None], profile=pf)
                    for pf in (False, True)]
        else:
            pair = [cb.prepare_device(D, S[None], lam, opt, mu=cfg["mu"],
                                      grd=(v == "cbpdngrd"), profile=pf)
                    for pf in (False, True)]
        solves.append((v, pair[0], pair[1]))

    def step(profiled=False):
        """One pass of every solve; with profiled, CUDA events around every
        kernel launch (the per-kernel split of the roofline)."""
        prof = {}
        for v, ds, dsp in solves:
            if not profiled:
                ds.run()
                continue
            dsp.run()
            for k, (ms, n) in dsp.profile().items():
                a = prof.setdefault(k, [0.0, 0])
                a[0] += ms
                a[1] += n
        return prof

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
    step(profiled=True)
    barrier()
    n_launch0 = _lib.sc_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        ev0.record()
        for _ in range(args.steps):
            step()
        ev1.record()
        barrier()
    ms = ev0.elapsed_time(ev1)
    launches = _lib.sc_launch_count() - n_launch0
    # the same steps again with an event pair around every kernel launch (on
    # the solver's stream): the per-kernel split and the roofline
    prof_tot = {}
    for _ in range(args.steps):
        for k, (pms, n) in step(profiled=True).items():
            a = prof_tot.setdefault(k, [0.0, 0])
            a[0] += pms
            a[1] += n
    barrier()
    iters_per_step = cfg["iters"] * len(cfg["variants"])
    value = replicas.job_rate(iters_per_step * args.steps, ms)
    ms = replicas.max_over_ranks(ms)

    # end to end through the reference-facing API (numpy host buffers in and
    # out, every host<->device copy inside the timed region)
    Dn = np.ascontiguousarray(np.moveaxis(Dh, 0, 2))

    def e2e_step():
        for v in cfg["variants"]:
            opt = opt_for(cfg, v)
            if v == "cbpdn":
                cb.cbpdn(Dn, Sh, lam, opt)
            elif v == "cbpdngrd":
                cb.cbpdngrd(Dn, Sh, lam, cfg["mu"], opt)
            else:
                cb.cbpdnmsk(Dn, Sh * maskh, maskh, lam, opt)
    if not args.no_e2e:
        e2e_step()
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        barrier()
        e_ms = (time.perf_counter() - t0) * 1e3
        e_value = replicas.job_rate(iters_per_step * args.steps, e_ms)
    else:
        e_value = None
    h2d = d2h = 0
    for v in cfg["variants"]:
        M = cfg["M"] + (1 if v == "cbpdnmsk" else 0)
        h2d += 4 * M * cfg["K"] ** 2 + 4 * cfg["H"] * cfg["W"] + 8  # D, S, scalars
        if v == "cbpdnmsk":
            h2d += 4 * cfg["H"] * cfg["W"] + 4 * M  # mask, l1 weights
        if v == "cbpdngrd":
            h2d += 4 * M
        d2h += 4 * M * cfg["H"] * cfg["W"]

    # roofline of one ADMM iteration (the timed solves' kernels)
    peak, peak_kind = measured_peaks()
    it_ms = sum(a[0] for a in prof_tot.values())
    n_it = prof_tot.get("col_kernel", [0, 1])[1]
    bytes_it = design_it = 0.0
    for v in cfg["variants"]:
        M = cfg["M"] + (1 if v == "cbpdnmsk" else 0)
        bytes_it += graded_bytes(cfg["H"], cfg["W"], M) * cfg["iters"] * args.steps
        design_it += design_bytes(cfg["H"], cfg["W"], M, v, cfg["K"]) * cfg["iters"] * args.steps
    # whole iterations as timed (launch gaps included); the per-kernel split
    # below comes from the profiled pass
    achieved = bytes_it / (ms / 1e3) / 1e9 if ms > 0 else None
    n_solve_it = cfg["iters"] * args.steps * len(cfg["variants"])
    kern = {k: {"ms_per_launch": a[0] / max(1, a[1]), "launches": a[1],
                "share": a[0] / it_ms if it_ms else None} for k, a in prof_tot.items()}
    # the dominant kernel: graded bytes per launch over its mean launch time
    dom = None
    if kern:
        name = max(kern, key=lambda k: kern[k]["ms_per_launch"] * kern[k]["launches"])
        gb = 0.0
        for v in cfg["variants"]:
            M = cfg["M"] + (1 if v == "cbpdnmsk" else 0)
            gb += graded_kernel_bytes(cfg["H"], cfg["W"], M).get(name, 0.0)
        gb /= len(cfg["variants"])
        t = kern[name]["ms_per_launch"]
        tr, src = MEASURED_TRAFFIC_PER_MAP.get((cfg["H"], cfg["W"]), {}).get(name, (None, None))
        dom = {"name": name, "share": kern[name]["share"],
               "algorithmic_bytes_per_launch": gb,
               "achieved": gb / (t / 1e3) / 1e9 if t > 0 and gb > 0 else None,
               "frac": gb / (t / 1e3) / 1e9 / peak if t > 0 and gb > 0 else None,
               "traffic": tr * cfg["M"] if tr else None,
               "traffic_source": src}

    # CPU baseline and relative error: the FP64 restatement's first n
    # iterations (rank 0 of a one-GPU run) against the same n iterations of
    # the device solver
    cpu = rel_err = None
    if rank == 0 and world == 1 and not args.no_cpu:
        n = cfg["check_iters"]
        cpu, ref = cpu_leg(cfg, Dh, Sh, maskh, n)
        from oracle import cbpdn_oracle_torch as OT
        rel_err = {"iterations": n, "X": {}, "functional": {}, "rho": {},
                   "reference": "FP64 CPU restatement, the same first %d iterations of the "
                                "same problem" % n}
        Dm = Dh.astype(np.float64)
        for v, ds, _ in solves:
            keep = ds.opts.max_iter
            ds.opts.max_iter = n
            Y = ds.run()[0]
            torch.cuda.synchronize()
            rho_gpu = ds.state()["rho"][0]
            ds.opts.max_iter = keep
            if v == "cbpdnmsk":
                Y = Y[1:]
            Yg = Y.cpu().numpy()
            Xo, info = ref[v]
            Yo = np.moveaxis(Xo, 2, 0)
            rel_err["X"][v] = float(np.linalg.norm((Yg - Yo).ravel()) /
                                    np.linalg.norm(Yo.ravel()))
            kw = {}
            if v == "cbpdngrd":
                kw = dict(mu=cfg["mu"], wgrd=np.ones(cfg["M"]))
            Ss = Sh
            if v == "cbpdnmsk":
                kw = dict(mask=maskh)
                Ss = Sh * maskh
            J = OT.objective(Dm, Ss, Yg, np.float32(lam), **kw)
            Jo = OT.objective(Dm, Ss, Yo, np.float32(lam), **kw)
            rel_err["functional"][v] = abs(J - Jo) / abs(Jo)
            rel_err["rho"][v] = abs(rho_gpu - info["rho"]) / info["rho"]
            del Y, Yg
    out = None
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "iter/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_dict(cfg, world),
            "e2e": {"value": e_value, "unit": "iter/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "hbm", "kernel": "ADMM iteration (col_kernel + row_kernel + "
                         "finalize_kernel + fixup_kernel)",
                         "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                         "unit": "GB/s", "frac": achieved / peak if achieved else None,
                         # DRAM bytes per launch of the dominant kernel (ncu)
                         "traffic": dom["traffic"] if dom else None,
                         "traffic_kernel": dom["name"] if dom and dom["traffic"] else None,
                         "algorithmic_bytes_per_iteration": bytes_it / n_solve_it,
                         "design_bytes_per_iteration": design_it / n_solve_it,
                         "design_frac": (design_it / (ms / 1e3) / 1e9 / peak)
                         if ms > 0 else None,
                         "iteration_ms": ms / n_solve_it,
                         "kernel_sum_ms_per_iteration": it_ms / max(1, n_it), "kernels": kern,
                         "dominant_kernel": dom},
            "rel_err": rel_err,
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
    return out


def synth_images(cfg, seed, device):
    """Config 2: uneven images from one dictionary, masks, lambdas (drawn on
    the device with torch; torch.fft for the synthesis only)."""
    import torch
    rng = np.random.default_rng(seed)
    M, K = cfg["M"], cfg["K"]
    g = torch.Generator(device=device).manual_seed(seed)
    D = torch.randn((M, K, K), generator=g, device=device)
    D /= torch.sqrt(torch.sum(D * D, dim=(1, 2), keepdim=True))
    imgs, masks = [], []
    for _ in range(cfg["nimg"]):
        H, W = (int(rng.choice(cfg["sides"])) for _ in range(2))
        Dp = torch.zeros((M, H, W), device=device)
        Dp[:, :K, :K] = D
        X0 = (torch.rand((M, H, W), generator=g, device=device) < cfg["density"]).float() * \
            torch.randn((M, H, W), generator=g, device=device)
        Sf = torch.sum(torch.fft.rfft2(Dp) * torch.fft.rfft2(X0), dim=0)
        S = torch.fft.irfft2(Sf, s=(H, W))
        S = S + 0.01 * torch.randn((H, W), generator=g, device=device)
        S = S - S.mean()
        p = float(rng.uniform(0.5, 0.9))
        mk = (torch.rand((H, W), generator=g, device=device) < p).float()
        imgs.append((S * mk).contiguous())
        masks.append(mk)
    lam = rng.uniform(0.02, 0.1, cfg["nimg"]).astype(np.float32)
    return D.contiguous(), imgs, masks, lam


def run_batched(args, cfg, rank, world, local_rank):
    """Config 2: image-iterations/s of the batched solver, and of a loop of
    single solves over the same images."""
    import torch
    import sporco_cuda.cbpdn as cb
    from sporco_cuda import _lib, replicas
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    D, imgs, masks, lam = synth_images(cfg, 12345 + args.config + rank, dev)
    Dk = D.permute(1, 2, 0).contiguous()
    opt = {"MaxMainIter": cfg["iters"], "RelStopTol": 1e-4, "AbsStopTol": 0.0,
           "RelaxParam": 1.8, "L1Weight": 1.0,
           "AutoRho": {"Enabled": True, "Period": 1, "Scaling": 1000.0, "RsdlRatio": 1.2,
                       "RsdlTarget": None, "AutoScaling": True, "StdResiduals": False}}

    def step():
        _, iters = cb.cbpdn_batched(Dk, imgs, lam, opt, W_list=masks, return_info=True)
        return iters

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
    barrier()
    n0 = _lib.sc_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    total_it = 0
    with ClockSampler(local_rank) as clk:
        ev0.record()
        for _ in range(args.steps):
            total_it += sum(step())
        ev1.record()
        barrier()
    ms = ev0.elapsed_time(ev1)
    launches = _lib.sc_launch_count() - n0
    value = replicas.job_rate(total_it, ms)
    ms = replicas.max_over_ranks(ms)
    # loop of single solves over the same images (device inputs)
    Di = torch.cat((torch.zeros((1, cfg["K"], cfg["K"]), device=dev), D), 0)
    Di[0, 0, 0] = 1.0  # the AMS impulse filter, as cbpdnmsk prepends it
    l1 = np.concatenate(([0.0], np.ones(cfg["M"]))).astype(F32)
    t0 = time.perf_counter()
    loop_it = 0
    for S, mk, lm in zip(imgs, masks, lam):
        ds = cb.prepare_device(Di, S[None], float(lm), opt, l1=l1, mask=mk.to(torch.int32)[None])
        ds.run()
        loop_it += ds.state()["iterations"][0]
    torch.cuda.synchronize()
    loop_ms = (time.perf_counter() - t0) * 1e3
    loop_value = loop_it / (loop_ms / 1e3)
    # end to end through the public API with numpy host buffers
    Dn = Dk.cpu().numpy()
    In = [x.cpu().numpy() for x in imgs]
    Wn = [x.cpu().numpy() for x in masks]
    barrier()
    t0 = time.perf_counter()
    out, e_iters = cb.cbpdn_batched(Dn, In, lam, opt, W_list=Wn, return_info=True)
    barrier()
    e_ms = (time.perf_counter() - t0) * 1e3
    e_value = sum(e_iters) / (e_ms / 1e3)
    h2d = 4 * Dn.size + sum(4 * x.size for x in In) + sum(4 * x.size for x in Wn) + 4 * len(lam)
    d2h = sum(4 * x.size for x in out)
    peak, peak_kind = measured_peaks()
    bytes_total = 0.0
    it_per_img = step()  # iteration counts per image (same data, same counts)
    bucket_it = {}
    for S, k in zip(imgs, it_per_img):
        H_, W_ = S.shape
        # state bytes per image-iteration; dictionary reads once per size and
        # iteration of its bucket (the longest-running image of that size)
        bytes_total += (graded_bytes(H_, W_, cfg["M"] + 1, 1) -
                        graded_bytes(H_, W_, cfg["M"] + 1, 0)) * k
        bucket_it[(H_, W_)] = max(bucket_it.get((H_, W_), 0), k)
    for (H_, W_), k in bucket_it.items():
        bytes_total += graded_bytes(H_, W_, cfg["M"] + 1, 0) * k
    achieved = bytes_total * args.steps / (ms / 1e3) / 1e9
    if rank != 0:
        return None
    shapes = sorted(set(tuple(x.shape) for x in imgs))
    return {
        "metric": METRIC, "value": value, "unit": "image-iter/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": cfg["workload"], "images": cfg["nimg"], "M": cfg["M"],
                   "K": cfg["K"], "buckets": len(shapes),
                   "parallelism": "replicas%d" % world if world > 1 else "single",
                   "l2": "working set larger than L2 (no flush)"},
        "loop_of_single_solves": {"value": loop_value, "unit": "image-iter/s",
                                  "speedup_batched_over_loop": value / loop_value},
        "e2e": {"value": e_value, "unit": "image-iter/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "hbm", "kernel": "batched solve (all buckets, all kernels)",
                     "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None},
        "iterations": {"mean": float(np.mean(it_per_img)), "max": int(np.max(it_per_img))},
        "cpu_baseline": None,
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }


def run_adjoint(args, cfg, rank, world, local_rank):
    """Config 3: forward + backward of the unrolled solve; image-iterations/s
    of forward+backward, and the backward/forward time ratio."""
    import torch
    import sporco_cuda.adjoint as adj
    import sporco_cuda.cbpdn as cb
    from sporco_cuda import _lib, replicas
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    B = cfg["nimg"]
    imgs = []
    D = None
    for b in range(B):
        Db, Sb, _ = synth(cfg, 12345 + args.config + 100 * b + 1000 * rank)
        if D is None:
            D = torch.from_numpy(Db).to(dev)
        imgs.append(torch.from_numpy(Sb).to(dev))
    # one dictionary for the batch: re-synthesise every clean image from D
    g = torch.Generator(device=dev).manual_seed(777 + rank)
    H, W, M, K = cfg["H"], cfg["W"], cfg["M"], cfg["K"]
    X0 = (torch.rand((B, H, W, M), generator=g, device=dev) < cfg["density"]).float() * \
        torch.randn((B, H, W, M), generator=g, device=dev)
    Dk = D.permute(1, 2, 0).contiguous()
    with torch.no_grad():
        Sc = adj.reconstruct(Dk, X0)
        Sc = Sc - Sc.mean(dim=(1, 2), keepdim=True)
    S = Sc + 0.05 * torch.randn((B, H, W), generator=g, device=dev)
    opt = {"MaxMainIter": cfg["iters"], "RelStopTol": 0.0, "RelaxParam": 1.8, "rho": None,
           "AutoRho": {"Enabled": False}}

    def fwd_bwd(checkpoints="sqrt"):
        Dg = Dk.clone().requires_grad_(True)
        Sg = S.clone().requires_grad_(True)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t2 = torch.cuda.Event(enable_timing=True)
        t0.record()
        X = adj.cbpdn_unrolled(Dg, Sg, cfg["lmbda"], opt, checkpoints=checkpoints)
        R = adj.reconstruct(Dg, X)
        L = torch.sum((R - Sc) ** 2) + 0.01 * torch.sum(torch.abs(X))
        t1.record()
        L.backward()
        t2.record()
        torch.cuda.synchronize()
        return t0.elapsed_time(t1), t1.elapsed_time(t2)

    for _ in range(args.warmup):
        fwd_bwd()
    torch.cuda.synchronize()
    n0 = _lib.sc_launch_count()
    f_ms = b_ms = 0.0
    with ClockSampler(local_rank) as clk:
        for _ in range(args.steps):
            f, b_ = fwd_bwd()
            f_ms += f
            b_ms += b_
    launches = _lib.sc_launch_count() - n0
    ms = f_ms + b_ms
    value = replicas.job_rate(B * cfg["iters"] * args.steps, ms)
    # every step's trace kept in the forward pass (no recomputation; about
    # K (R + C) bytes of workspace), for comparison
    fwd_bwd("all")
    torch.cuda.synchronize()
    fa = ba = 0.0
    for _ in range(args.steps):
        f, b_ = fwd_bwd("all")
        fa += f
        ba += b_
    fa = replicas.max_over_ranks(fa)
    ba = replicas.max_over_ranks(ba)
    f_ms = replicas.max_over_ranks(f_ms)
    b_ms = replicas.max_over_ranks(b_ms)
    ms = f_ms + b_ms
    # the fused solver on the same batch, for reference
    ds = cb.prepare_device(D, S, cfg["lmbda"], opt)
    ds.run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    ds.run()
    e1.record()
    torch.cuda.synchronize()
    fused_ms = e0.elapsed_time(e1)
    peak, peak_kind = measured_peaks()
    if rank != 0:
        return None
    # the forward's graded bytes over its device time (K iterations of B images)
    fwd_bytes = graded_bytes(H, W, M, B) * cfg["iters"]
    f_step = f_ms / args.steps
    roof = {"bound": "hbm", "kernel": "unrolled forward (K ADMM iterations, B images)",
            "achieved": fwd_bytes / (f_step / 1e3) / 1e9, "peak": peak, "peak_kind": peak_kind,
            "unit": "GB/s", "frac": fwd_bytes / (f_step / 1e3) / 1e9 / peak, "traffic": None,
            "fused_forward_frac": fwd_bytes / (fused_ms / 1e3) / 1e9 / peak}
    cpu = rel = None
    if world == 1 and not args.no_cpu:
        cpu, rel = adjoint_cpu_leg(cfg, Dk[..., :].float(), S[0], Sc[0])
    return {
        "metric": METRIC, "value": value, "unit": "image-iter/s (forward+backward)",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": cfg["workload"], "images": B, "H": H, "W": W, "M": M, "K": K,
                   "iterations": cfg["iters"], "checkpoints": "every ceil(sqrt(K)) iterations",
                   "l2": "working set larger than L2 (no flush)"},
        "forward_ms": f_ms / args.steps, "backward_ms": b_ms / args.steps,
        "backward_over_forward": b_ms / f_ms,
        "fused_forward_solve_ms": fused_ms,
        "backward_over_fused_forward": (b_ms / args.steps) / fused_ms,
        "all_traces": {"forward_ms": fa / args.steps, "backward_ms": ba / args.steps,
                       "backward_over_forward": ba / fa,
                       "backward_over_fused_forward": (ba / args.steps) / fused_ms,
                       "checkpoints": "every step's trace kept in the forward pass"},
        "e2e": None, "roofline": roof, "rel_err": rel, "cpu_baseline": cpu,
        "gpu_launches": launches, "clocks": clk.summary(),
    }


def adjoint_cpu_leg(cfg, Dk, S1, Sc1, iters=10):
    """Config 3 on the host: torch FP64 autograd of the plain unrolled solve
    (the adjoint oracle) for one image and `iters` iterations, timed
    (forward + backward), and the GPU adjoint's gradients on the same sample
    against it: against the FP64 loss along the GPU forward's own shrinkage
    pattern (a float32 and a float64 forward can put a near-threshold
    element on different sides of its kink), and against the plain FP64
    gradient, with the number of elements whose pattern differs."""
    import torch
    import sporco_cuda.adjoint as adj
    from oracle import adjoint_oracle as A
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    lam = float(np.float32(cfg["lmbda"]))
    rho = float(np.float32(50 * lam + 1))
    alpha = float(np.float32(1.8))
    Sc64 = Sc1.detach().double().cpu()[None]
    Dd = Dk.detach().double().cpu().requires_grad_(True)
    Sd = S1.detach().double().cpu()[None].requires_grad_(True)
    trace = []
    t0 = time.perf_counter()
    Y64 = A.unrolled(Dd, Sd, lam, rho, alpha, iters, trace=trace)
    L = torch.sum((A.reconstruct(Dd, Y64) - Sc64) ** 2) + 0.01 * torch.sum(torch.abs(Y64))
    L.backward()
    dt = time.perf_counter() - t0
    cpu = {"value": iters / dt, "unit": "image-iter/s (forward+backward)", "cores": threads,
           "kind": "port",
           "sample": "one %dx%d image, M=%d, %d unrolled iterations: FP64 torch autograd of the "
                     "unrolled restatement (%d threads)" % (cfg["H"], cfg["W"], cfg["M"], iters,
                                                          threads)}
    opt = {"MaxMainIter": iters, "RelStopTol": 0.0, "RelaxParam": 1.8, "rho": None,
           "AutoRho": {"Enabled": False}}
    Dg = Dk.detach().clone().requires_grad_(True)
    Sg = S1.detach()[None].clone().requires_grad_(True)
    X = adj.cbpdn_unrolled(Dg, Sg, cfg["lmbda"], opt)
    R = adj.reconstruct(Dg, X)
    Lg = torch.sum((R - Sc1[None]) ** 2) + 0.01 * torch.sum(torch.abs(X))
    Lg.backward()
    masks = []
    for k in range(1, iters + 1):
        Xk = adj.cbpdn_unrolled(Dk.detach(), S1.detach()[None], cfg["lmbda"],
                                dict(opt, MaxMainIter=k))
        masks.append((Xk != 0).permute(0, 3, 1, 2).cpu())
    flips = int(sum(int(torch.sum((y != 0) != m)) for y, m in zip(trace, masks)))
    Dm = Dk.detach().double().cpu().requires_grad_(True)
    Sm = S1.detach().double().cpu()[None].requires_grad_(True)
    A.loss(Dm, Sm, Sc64, lam, rho, alpha, iters, 0.01, masks=masks).backward()

    def r(a, b):
        return float(torch.linalg.norm(a.double().cpu() - b) / torch.linalg.norm(b))
    rel = {"iterations": iters, "images": 1,
           "gD": r(Dg.grad, Dm.grad), "gS": r(Sg.grad, Sm.grad),
           "reference": "FP64 torch autograd of the unrolled restatement along the GPU "
                        "forward's shrinkage pattern",
           "gD_plain": r(Dg.grad, Dd.grad), "gS_plain": r(Sg.grad, Sd.grad),
           "pattern_differences": flips}
    return cpu, rel


def run_reference(args, cfg, rank, world):
    """The reference algorithm's CPU implementation on this host's cores: the
    FP64 restatement (the reference ships no CPU solver; sporco, whose
    ConvBPDN it mirrors, is not installed), torch on every host thread, maps
    in chunks.  Each step continues one solve of the workload by a bounded
    number of iterations (SC_REF_STEP_SECONDS, default 8 s, at least one
    iteration).  Nothing of this package is loaded."""
    if rank != 0:
        return None
    if args.config in (2, 3):
        return {"impl": "reference",
                "unavailable": "the CPU restatement is timed on the single-solve workloads "
                               "(configs 0, 1, 4) only"}
    import torch
    from oracle import cbpdn_oracle_torch as OT
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    D, S, mask = synth(cfg, 12345 + args.config)
    budget = float(os.environ.get("SC_REF_STEP_SECONDS", "8"))
    gens = []
    for v in cfg["variants"]:
        a = _oracle_args(cfg, v, D, S, mask, cfg["iters"])
        a.pop("variant")
        prob, res, xi = OT.problem(v, **a)
        gens.append(OT.iterate(prob, res, xi, record=False))
    per_it = None
    times, counts = [], []
    done = 0
    for i in range(args.warmup + args.steps):
        n = 1 if per_it is None else max(1, int(budget / per_it))
        n = max(1, min(n, cfg["iters"] - done))
        t0 = time.perf_counter()
        for _ in range(n):
            for gen in gens:
                next(gen, None)
        dt = time.perf_counter() - t0
        done += n
        if i > 0 or per_it is None:
            per_it = dt / n
        if i >= args.warmup:
            times.append(dt)
            counts.append(n * len(gens))
        if done >= cfg["iters"]:  # the solve is over: start it again
            gens = []
            for v in cfg["variants"]:
                a = _oracle_args(cfg, v, D, S, mask, cfg["iters"])
                a.pop("variant")
                prob, res, xi = OT.problem(v, **a)
                gens.append(OT.iterate(prob, res, xi, record=False))
            done = 0
    value = sum(counts) / sum(times)
    ref_gpu = reference_gpu_leg(args, cfg, D, S, mask)
    sample = ("%s: %d timed steps of one continuing FP64 solve (%d ADMM iterations of %s in "
              "all, set-up in the untimed warm-up; torch CPU, %d threads, maps in chunks of 16)"
              % (cfg["workload"], args.steps, sum(counts), " and ".join(cfg["variants"]),
                 threads))
    return {
        "metric": METRIC, "value": value, "unit": "iter/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": config_dict(cfg, world),
        "cpu_baseline": {"value": value, "unit": "iter/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "iter/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "reference_gpu": ref_gpu,
    }


def reference_gpu_leg(args, cfg, D, S, mask):
    """The reference's own CUDA implementation of the path (its sources,
    unchanged, built for sm_100a into oracle/_ref by oracle/Makefile) on the
    same workload, through its own C ABI with host buffers: every call plans
    its FFTs, allocates, copies in, runs its host-driven iterations and
    copies out, as a caller of the reference sees it.  Its default
    HighMemSolve = 0 (its fastest mode; its solve coefficients then go
    stale after a change of rho).  One untimed call per variant, then timed
    calls for at most about 30 s."""
    try:
        import torch
        if not torch.cuda.is_available():
            return {"unavailable": "no CUDA device"}
        from oracle import ref_abi
    except Exception as e:  # pragma: no cover
        return {"unavailable": "reference build not importable: %s" % e}
    if not ref_abi.available():
        return {"unavailable": "oracle/_ref not built (make -C oracle ref REF=<reference tree>)"}
    Dk = np.ascontiguousarray(np.moveaxis(D, 0, 2))

    def call(v):
        opt = dict(opt_for(cfg, v), AuxVarObj=False, HighMemSolve=False, NonNegCoef=False,
                   NoBndryCross=False)
        if v == "cbpdn":
            ref_abi.cbpdn(Dk, S, cfg["lmbda"], opt)
        elif v == "cbpdngrd":
            ref_abi.cbpdngrd(Dk, S, cfg["lmbda"], cfg["mu"], opt)
        else:
            ref_abi.cbpdnmsk(Dk, S * mask, mask, cfg["lmbda"], opt)
    for v in cfg["variants"]:
        call(v)
    n, t0 = 0, time.perf_counter()
    while n < max(1, args.steps):
        for v in cfg["variants"]:
            call(v)
        n += 1
        if time.perf_counter() - t0 > 30.0:
            break
    dt = time.perf_counter() - t0
    iters = n * cfg["iters"] * len(cfg["variants"])
    return {"value": iters / dt, "unit": "iter/s", "calls": n * len(cfg["variants"]),
            "ms_per_call": 1e3 * dt / (n * len(cfg["variants"])),
            "kind": "the reference's CUDA sources built for sm_100a (oracle/_ref), its C ABI "
                    "with host buffers (set-up, copies and %d iterations per call; "
                    "HighMemSolve off)" % cfg["iters"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", type=int, default=DEFAULT_CONFIG, choices=sorted(CONFIGS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end arm")
    ap.add_argument("--iters", type=int, default=0,
                    help="override the iterations per solve (profiling runs only)")
    args = ap.parse_args()
    cfg = dict(CONFIGS[args.config])
    if args.iters > 0:
        cfg["iters"] = args.iters
        cfg["workload"] += " [cut to %d iterations]" % args.iters
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        out = run_reference(args, cfg, rank, world)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.config == 2:
        out = run_batched(args, cfg, rank, world, local_rank)
    elif args.config == 3:
        out = run_adjoint(args, cfg, rank, world, local_rank)
    else:
        out = run_ours(args, cfg, rank, world, local_rank)
    if out is not None:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
