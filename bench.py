"""Benchmark of the MKF hot path on B200: scalar field -> K binary pattern distributions.

Workload (N=1): a 1024^3 FP64 Gaussian random field (N(0,1) white noise from a fixed seed,
periodic Gaussian smoothing sigma = 4 voxels, renormalised to zero mean / unit variance) with 16
thresholds evenly spaced in [-2, 2], relation '>'. One step = one read of the field giving 16
distributions (mkfFieldBPFD) plus their Minkowski measures on the device (mkfMeasuresF64Dev).
Inputs are 8.6 GB, far larger than the 126 MB L2, so no flush is needed between steps.

  value     Gvoxel/s with the field resident in HBM (device-timed, max over ranks)
  e2e       Gvoxel/s through the host-buffer entry point mkfFieldBPFDHost: each step copies the
            pinned host field to the GPU (slabs overlapped with counting) and the counts back
  roofline  the fused kernel's algorithmic bytes / its CUDA-event time vs measured HBM peak
  cpu_baseline  the reference MKF C path (compiled from its sources) on this host's cores over the
            whole field; its counts must equal the timed counts (counts_equal_reference); beside
            it the reference's single-thread entry point on a 16-plane slab

With torchrun (N > 1) every rank counts its own 1024^3 slab (1025 planes: one halo plane) of a
field sharded along z through mkf_b200.shard.sharded_field_bpfd, which sums the 16 x 256 partial
counts with an NCCL all-reduce each step (weak scaling). `--impl reference` times the reference C path alone (rank 0) and, as a
second reference point under "reference_cuda", the reference's own CUDA path compiled for sm_100a.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

N_SIDE = 1024
SIGMA = 4.0
K_THRESH = 16
THRESHOLDS = np.linspace(-2.0, 2.0, K_THRESH)
SEED = 20261203
WORKLOAD = "grf1024_f64_k16"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="mkf", choices=["mkf", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true", help="skip the batched, serving and in-situ workloads (and the reference CUDA point of the reference arm)")
    ap.add_argument("--profile", choices=["field", "batch", "planewave", "dropin"], default=None,
                    help="run one small case for a profiler instead of the benchmark: 'field' = one "
                         "GRF (--side, --dtype, --thresholds), 'batch' = the uneven ball batch (--fields), "
                         "'planewave' = one 1024 x 1024 x --side FP32 step of the in-situ series, "
                         "thresholds {-0.5, 0, 0.5}, 'dropin' = the drop-in pair binMapCUDA + "
                         "mkfCUDAGetBPFD on the 256^3 FP32 ball, threshold 0")
    ap.add_argument("--side", type=int, default=512)
    ap.add_argument("--dtype", choices=["f32", "f64"], default="f64")
    ap.add_argument("--thresholds", default="16", help="a count n (linspace(-2, 2, n)) or a comma list of values")
    ap.add_argument("--fields", type=int, default=128)
    ap.add_argument("--reps", type=int, default=2)
    return ap.parse_args()


# ---------------------------------------------------------------- synthetic fields

def grf_torch(nz, ny, nx, seed, device):
    """Gaussian random field on the GPU (FFT smoothing), FP64, zero mean, unit variance."""
    import torch

    g = torch.Generator(device=device).manual_seed(seed)
    w = torch.randn((nz, ny, nx), dtype=torch.float64, device=device, generator=g)
    W = torch.fft.rfftn(w)
    del w
    two_pi = 2 * math.pi
    for dim, n in ((0, nz), (1, ny)):
        k = torch.fft.fftfreq(n, device=device, dtype=torch.float64) * two_pi
        shape = [1, 1, 1]
        shape[dim] = n
        W *= torch.exp(-0.5 * SIGMA * SIGMA * k * k).view(shape)
    kx = torch.fft.rfftfreq(nx, device=device, dtype=torch.float64) * two_pi
    W *= torch.exp(-0.5 * SIGMA * SIGMA * kx * kx).view(1, 1, -1)
    f = torch.fft.irfftn(W, s=(nz, ny, nx))
    del W
    f -= f.mean()
    f /= f.std()
    torch.cuda.synchronize(device)
    return f.contiguous()


def grf_numpy(nz, ny, nx, seed):
    """The same kind of field on the host (for the reference arm), flattened. X = 1024 is a
    multiple of 32, so the reference CPU map reads nothing past the end."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((nz, ny, nx))
    W = np.fft.rfftn(w)
    del w
    two_pi = 2 * math.pi
    kz = np.fft.fftfreq(nz) * two_pi
    ky = np.fft.fftfreq(ny) * two_pi
    kx = np.fft.rfftfreq(nx) * two_pi
    W *= np.exp(-0.5 * SIGMA * SIGMA * kz * kz)[:, None, None]
    W *= np.exp(-0.5 * SIGMA * SIGMA * ky * ky)[None, :, None]
    W *= np.exp(-0.5 * SIGMA * SIGMA * kx * kx)[None, None, :]
    f = np.fft.irfftn(W, s=(nz, ny, nx), axes=(0, 1, 2))
    f -= f.mean()
    f /= f.std()
    return np.ascontiguousarray(f.ravel())


def ball_field(shape_zyx, rng, g, device, dtype):
    """Max over 1-64 balls (centres uniform in the box, radii uniform in [2, 40]) of r - |x - c|,
    plus N(0, 0.1) noise. The max is formed inside each ball's bounding box only: elsewhere the
    value stays far below zero, which maps the same at thresholds near 0."""
    import torch

    Z, Y, X = shape_zyx
    f = torch.full((Z, Y, X), -50.0, dtype=dtype, device=device)
    for _b in range(int(rng.integers(1, 65))):
        c = rng.random(3) * np.array([X, Y, Z])
        r = float(rng.uniform(2, 40))
        lo3 = [max(0, int(np.floor(c[i] - r - 1))) for i in range(3)]
        hi3 = [min((X, Y, Z)[i], int(np.ceil(c[i] + r + 2))) for i in range(3)]
        if min(hi3[i] - lo3[i] for i in range(3)) <= 0:
            continue
        zz = torch.arange(lo3[2], hi3[2], device=device, dtype=dtype).view(-1, 1, 1) - c[2]
        yy = torch.arange(lo3[1], hi3[1], device=device, dtype=dtype).view(1, -1, 1) - c[1]
        xx = torch.arange(lo3[0], hi3[0], device=device, dtype=dtype).view(1, 1, -1) - c[0]
        v = r - torch.sqrt(zz * zz + yy * yy + xx * xx)
        box = f[lo3[2]:hi3[2], lo3[1]:hi3[1], lo3[0]:hi3[0]]
        torch.maximum(box, v, out=box)
    f.add_(torch.randn((Z, Y, X), dtype=dtype, device=device, generator=g).mul_(0.1))
    return f


def ball_fields(n_fields, seed, device, lo=17, hi=400, dtype=None):
    """The uneven batch: each axis uniform in [lo, hi], ball content (ball_field)."""
    import torch

    dtype = dtype or torch.float32
    rng = np.random.default_rng(seed)
    g = torch.Generator(device=device).manual_seed(seed)
    fields = []
    for _ in range(n_fields):
        X, Y, Z = (int(v) for v in rng.integers(lo, hi + 1, size=3))
        fields.append(ball_field((Z, Y, X), rng, g, device, dtype))
    torch.cuda.synchronize(device)
    return fields


def run_batch_workload(dev, n_fields=512, seed=SEED + 3, reps=3):
    """Uneven batch (512 FP32 fields, threshold 0): fields/s of the plain drop-in call per field
    (binMapCUDA + mkfCUDAGetBPFDH), of the fused call per field (mkfFieldBPFD), and of one
    batched launch (mkfBatchPlanLaunch, and replayed as a CUDA graph)."""
    import torch

    import mkf_b200

    fields = ball_fields(n_fields, seed, dev)
    vox = sum(f.numel() for f in fields)
    t = [0.0]
    # plain drop-in: one map + one count + one host copy per field, synchronous
    mkf_b200.get_bpfd_host(*mkf_b200.bin_map_cuda(fields[0], ">", 0.0)[:2])
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for f in fields:
        pbm, org, _ = mkf_b200.bin_map_cuda(f, ">", 0.0)
        mkf_b200.get_bpfd_host(pbm, org)
    plain_s = time.perf_counter() - t0
    # fused per field (asynchronous calls, one synchronisation at the end)
    outs = [torch.zeros((1, 256), dtype=torch.int64, device=dev) for _ in fields]
    for f, o in zip(fields, outs):
        mkf_b200.field_bpfd(f, t, mkf_b200.BMC_GT, out=o)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for f, o in zip(fields, outs):
        mkf_b200.field_bpfd(f, t, mkf_b200.BMC_GT, out=o)
    e1.record()
    torch.cuda.synchronize(dev)
    fused_s = e0.elapsed_time(e1) * 1e-3
    # batched: one launch (and a CUDA graph replay) for all fields
    plan = mkf_b200.BatchPlan(fields, [t] * len(fields))
    plan.launch()
    plan.launch_graph()
    torch.cuda.synchronize(dev)
    times = {}
    for name, fn in (("batched", plan.launch), ("batched_graph", plan.launch_graph)):
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize(dev)
        times[name] = e0.elapsed_time(e1) * 1e-3 / reps
    # the batched counts equal the per-field ones
    same = bool(torch.equal(plan.out, torch.cat(outs)))
    plan.close()
    res = {
        "workload": f"{n_fields} FP32 fields, axes U[17,400], balls + N(0,0.1) noise, threshold 0 (>)",
        "voxels": int(vox),
        "plain_dropin_fields_per_s": n_fields / plain_s,
        "fused_per_field_fields_per_s": n_fields / fused_s,
        "batched_fields_per_s": n_fields / times["batched"],
        "batched_graph_fields_per_s": n_fields / times["batched_graph"],
        "batched_gvoxel_per_s": vox / times["batched"] * 1e-9,
        "batched_vs_plain": plain_s / times["batched"],
        "batched_equals_per_field": same,
    }
    del fields, outs
    torch.cuda.empty_cache()
    return res


def serving_pool(dev, n=256, seed=SEED + 4):
    """Distinct fields a serving run draws from (requests cycle through them in a shuffled order,
    so no field repeats within n requests): voxel counts log-uniform in [32^3, 512^3], aspect
    ratios up to 4:1, 70 % FP32 / 30 % FP64, ball content; even entries stay on the device, odd
    ones are pinned host copies (the server stages those). 256 fields hold about 20 GB."""
    import torch

    rng = np.random.default_rng(seed)
    g = torch.Generator(device=dev).manual_seed(seed)
    pool = []
    for i in range(n):
        vox = float(np.exp(rng.uniform(np.log(32.0 ** 3), np.log(512.0 ** 3))))
        a = np.exp(rng.uniform(-np.log(2.0), np.log(2.0), size=3))  # max / min <= 4
        a = a / np.cbrt(a.prod())
        X, Y, Z = (max(2, int(round(np.cbrt(vox) * v))) for v in a)
        dt = torch.float32 if rng.random() < 0.7 else torch.float64
        f = ball_field((Z, Y, X), rng, g, dev, dt)
        if i % 2:
            h = torch.empty(f.shape, dtype=dt, pin_memory=True)
            h.copy_(f)
            del f
            f = h
        pool.append(f)
    torch.cuda.synchronize(dev)
    return pool


def run_plain_workload(dev, steps=20, warmup=5):
    """The plain method's workload (256^3 FP32 ball, threshold 0, '>'), field resident in HBM, L2
    flushed before each call (the field is 67 MB, inside the 126 MB L2):

    * fused: mkfFieldBPFD, CUDA events around each call with the queue kept busy (device time)
      and with a synchronize after each call (the latency a caller sees through the Python API);
    * dropin_pair: binMapCUDA + mkfCUDAGetBPFD called through the C ABI with their arguments built
      once, as a C caller of the original makes them; time per pair including the host
      synchronisation the original's per-stage timers impose, and the two stage times the
      library reports in KernInfo (the same quantities the reference CUDA point reports)."""
    import ctypes as C

    import torch

    import mkf_b200
    from mkf_b200 import _lib

    f = ball256_torch(dev)
    n = f.numel()
    Z, Y, X = f.shape
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(128 << 20, dtype=torch.int32, device=dev)  # 512 MB
    out = torch.zeros((1, 256), dtype=torch.int64, device=dev)
    res = {"workload": "256^3 FP32 ball (100 - |x - c| + U[-0.5, 0.5) noise), threshold 0, '>'",
           "l2": "flushed before each call"}

    def fused():
        mkf_b200.field_bpfd(f, [0.0], mkf_b200.BMC_GT, out=out, stream=stream)

    for _ in range(warmup):
        fused()
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for e0, e1 in ev:
        flush.zero_()
        e0.record(stream)
        fused()
        e1.record(stream)
    torch.cuda.synchronize(dev)
    dev_ms = float(np.median([e0.elapsed_time(e1) for e0, e1 in ev]))
    api = []
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        fused()
        torch.cuda.synchronize(dev)
        api.append((time.perf_counter() - t0) * 1e3)
    api_ms = float(np.median(api))
    res["fused"] = {"device_ms_per_call": dev_ms, "gvoxel_per_s": n / dev_ms * 1e-6, "api_ms_per_call": api_ms}

    L = mkf_b200.lib()
    defs = (C.c_int * 3)(X, Y, Z)
    table = (_lib.ConstFieldPtr * 4)()
    table[0].p = f.data_ptr()
    fi = _lib.BMFieldInfo()
    fi.fieldTableMask = 1
    fi.elemID = _lib.ENC_F32
    fi.profID = 0
    fi.pD = defs
    fi.pFieldDevPtrTable = table
    bm = _lib.BinMapF64()
    L.setBinMapF64(C.byref(bm), b">", 0.0)
    org = _lib.BMOrg()
    ki = _lib.KernInfo()
    pbm = torch.empty(int(L.setBMO(None, defs, bytes([0]))), dtype=torch.int32, device=dev)

    def pair():
        if not L.binMapCUDA(C.byref(ki), pbm.data_ptr(), C.byref(org), C.byref(fi), C.byref(bm)):
            raise RuntimeError("binMapCUDA returned NULL")
        L.mkfCUDAGetBPFD(C.byref(ki), out.data_ptr(), C.byref(org), pbm.data_ptr(), _lib.MKFCU_PROFILE_FAST)
        return ki.dtms[0], ki.dtms[1]

    for _ in range(warmup):
        pair()
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    t_map = t_cnt = 0.0
    for e0, e1 in ev:
        flush.zero_()
        e0.record(stream)
        a, b = pair()
        e1.record(stream)
        t_map += a
        t_cnt += b
    torch.cuda.synchronize(dev)
    ms = float(np.median([e0.elapsed_time(e1) for e0, e1 in ev]))
    res["dropin_pair"] = {"ms_per_pair": ms, "gvoxel_per_s": n / ms * 1e-6, "map_ms": t_map / steps,
                          "bpfd_ms": t_cnt / steps}
    del f, flush, pbm
    torch.cuda.empty_cache()
    return res


def run_serving_workload(dev, rates=(100, 500, 1000, 2000, 5000), max_requests=10000, seconds=3.0,
                         seed=SEED + 5):
    """Poisson request streams at each rate (min(10000, rate x 3 s) requests, so every rate runs a
    few seconds): each request takes the next field of a shuffled cycle through the pool and 1-8
    thresholds in [-2, 2] (relation >), counts stay on the device until the client has waited for
    them and released them. Reports p50/p99 latency (submission to completion) and throughput per
    rate, the saturated throughput (every request submitted at once), the device time of the
    launches and the worker's host planning time, the same device-resident requests as one batch
    plan (the kernels alone), and the plain per-field drop-in call on the same mix."""
    import threading

    import torch

    import mkf_b200

    pool = serving_pool(dev)
    rng = np.random.default_rng(seed)
    srv = mkf_b200.Server(hbm_budget=64 << 30)

    cursor = [0, rng.permutation(len(pool))]

    def requests(n):
        idx = []
        for _ in range(n):  # a shuffled cycle through the pool: distinct fields within a cycle
            if cursor[0] == len(pool):
                cursor[0], cursor[1] = 0, rng.permutation(len(pool))
            idx.append(int(cursor[1][cursor[0]]))
            cursor[0] += 1
        ks = rng.integers(1, 9, size=n)
        return [(i, np.sort(rng.uniform(-2, 2, size=int(k)))) for i, k in zip(idx, ks)]

    def stream(reqs, rate):
        gaps = rng.exponential(1.0 / rate, size=len(reqs)) if rate else np.zeros(len(reqs))
        tickets = [None] * len(reqs)
        done = threading.Event()

        def waiter():
            for j in range(len(reqs)):
                while tickets[j] is None:
                    time.sleep(0.0001)
                srv.wait(tickets[j], timeout=600)
                srv.release(tickets[j])
            done.set()

        w = threading.Thread(target=waiter)
        w.start()
        t0 = time.perf_counter()
        due = t0
        for j, (i, t) in enumerate(reqs):
            due += gaps[j]
            while True:
                now = time.perf_counter()
                if now >= due:
                    break
                if due - now > 0.0003:
                    time.sleep(due - now - 0.0002)
            tickets[j] = srv.submit(pool[i], t, mkf_b200.BMC_GT)
        done.wait()
        t1 = time.perf_counter()
        w.join()
        st = srv.stats(reset=True)
        vox = sum(pool[i].numel() for i, _ in reqs)
        h2d = sum(pool[i].numel() * pool[i].element_size() for i, _ in reqs if not pool[i].is_cuda)
        return {"requests": len(reqs), "offered_per_s": rate, "fields_per_s": len(reqs) / (t1 - t0),
                "gvoxel_per_s": vox / (t1 - t0) * 1e-9, "h2d_gb_per_s": h2d / (t1 - t0) * 1e-9,
                "p50_ms": st["p50"] * 1e3, "p99_ms": st["p99"] * 1e3,
                "launches": st["launches"], "mean_fields_per_launch": st["meanFieldsInLaunch"],
                "launch_device_s": st["launchDeviceSec"], "plan_host_s": st["planHostSec"], "wall_s": t1 - t0}

    stream(requests(200), 0)  # warm-up
    per_rate = [stream(requests(int(min(max_requests, r * seconds))), r) for r in rates]
    burst = stream(requests(2000), 0)
    dev_only = [r for r in requests(6000) if pool[r[0]].is_cuda][:2000]
    burst_dev = stream(dev_only, 0)
    # the kernels alone on the same device-resident mix: 128 of those requests on distinct fields
    # as one batch plan, against the server running the same requests
    head, seen = [], set()
    for r in dev_only:
        if r[0] not in seen and len(head) < 128:
            seen.add(r[0])
            head.append(r)
    plan = mkf_b200.BatchPlan([pool[i] for i, _ in head], [t for _, t in head])
    plan.launch()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(3):
        plan.launch()
    e1.record()
    torch.cuda.synchronize(dev)
    plan_s = e0.elapsed_time(e1) * 1e-3 / 3
    plan.close()
    head_vox = sum(pool[i].numel() for i, _ in head)
    served_head = stream(head, 0)

    # the plain per-field call on a sample of the same mix: host fields copied first, then one
    # binMapCUDA + mkfCUDAGetBPFDH per threshold, as a caller of the original library would
    sample = requests(100)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for i, t in sample:
        f = pool[i] if pool[i].is_cuda else pool[i].to(dev, non_blocking=True)
        for tv in t:
            pbm, org, _ = mkf_b200.bin_map_cuda(f, ">", float(tv))
            mkf_b200.get_bpfd_host(pbm, org)
    plain = len(sample) / (time.perf_counter() - t0)
    srv.close()
    del pool
    torch.cuda.empty_cache()
    return {
        "workload": "Poisson requests, voxels log-uniform 32^3..512^3, aspect <= 4:1, 70% FP32, 1-8 thresholds, "
                    "half device / half pinned host, 64 GB budget",
        "per_rate": per_rate,
        "saturated_fields_per_s": burst["fields_per_s"],
        "saturated_h2d_gb_per_s": burst["h2d_gb_per_s"],
        "saturated_device_resident_fields_per_s": burst_dev["fields_per_s"],
        "saturated_device_resident_gvoxel_per_s": burst_dev["gvoxel_per_s"],
        "saturated_device_resident_p99_ms": burst_dev["p99_ms"],
        "saturated_device_resident_launch_device_s": burst_dev["launch_device_s"],
        "saturated_device_resident_plan_host_s": burst_dev["plan_host_s"],
        "saturated_device_resident_wall_s": burst_dev["wall_s"],
        "device_resident_128_batch_plan_gvoxel_per_s": head_vox / plan_s * 1e-9,
        "device_resident_128_served_gvoxel_per_s": served_head["gvoxel_per_s"],
        "device_resident_128_served_launch_device_s": served_head["launch_device_s"],
        "device_resident_128_served_wall_s": served_head["wall_s"],
        "bound": "host-to-device copies of the pinned-host half of the requests (PCIe) at saturation",
        "saturated_p99_ms": burst["p99_ms"],
        "plain_dropin_fields_per_s": plain,
        "saturated_vs_plain": burst["fields_per_s"] / plain,
    }


def plane_wave_field(out, n_waves, seed, step, chunk=16):
    """Fill `out` (Z, Y, X) FP32 on the GPU with the in-situ series at time step `step`: a sum of
    n_waves plane waves (unit-norm random directions, |k| uniform in [0.05, 0.1] rad/voxel, phases
    from the seed, each advanced by its own rotation per step), scaled to unit variance. Plane z
    is Re((A_y * a_z) @ A_x^T) with A_x[x, w] = exp(i k_x,w x): batched complex GEMMs."""
    import torch

    dev = out.device
    rng = np.random.default_rng(seed)
    d = rng.standard_normal((n_waves, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    kv = d * rng.uniform(0.05, 0.1, size=n_waves)[:, None]
    ph = rng.uniform(0, 2 * np.pi, size=n_waves) + step * rng.uniform(-0.3, 0.3, size=n_waves)
    Z, Y, X = out.shape
    k = torch.tensor(kv, dtype=torch.float64, device=dev)
    ax = torch.exp(1j * torch.arange(X, dtype=torch.float64, device=dev)[:, None] * k[None, :, 0]).to(torch.complex64)
    ay = torch.exp(1j * torch.arange(Y, dtype=torch.float64, device=dev)[:, None] * k[None, :, 1]).to(torch.complex64)
    phase = torch.tensor(ph, dtype=torch.float64, device=dev)
    scale = float(np.sqrt(2.0 / n_waves))
    for z0 in range(0, Z, chunk):
        z = torch.arange(z0, min(Z, z0 + chunk), dtype=torch.float64, device=dev)
        az = torch.exp(1j * (z[:, None] * k[None, :, 2] + phase[None, :])).to(torch.complex64)
        out[z0:z0 + len(z)] = torch.matmul(ay[None] * az[:, None, :], ax.T).real * scale
    torch.cuda.synchronize(dev)


def run_insitu_workload(dev, steps=20, streamed_steps=3, shape=(1536, 2048, 2048), seed=SEED + 6):
    """The large in-situ series (2048 x 2048 x 1536 FP32, 25.8 GB), thresholds {-0.5, 0, 0.5}: all
    20 time steps counted device-resident (the field in HBM, refilled by the generator each step;
    CUDA events around the count), and the first `streamed_steps` of them also streamed from pinned
    host memory through mkfFieldBPFDHost (wall clock, host -> device copies overlapped with
    counting: about 0.5 s of PCIe per step, so not every step), with the same counts."""
    import torch

    import mkf_b200

    t = [-0.5, 0.0, 0.5]
    f = torch.empty(shape, dtype=torch.float32, device=dev)
    h = torch.empty(shape, dtype=torch.float32, pin_memory=True)
    vox = f.numel()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dev_ms, host_s, same = [], [], True
    out = None
    for step in range(steps):
        plane_wave_field(f, 256, seed, step)
        if out is None:
            out = mkf_b200.field_bpfd(f, t, mkf_b200.BMC_GT)  # warm-up
        out.zero_()
        e0.record()
        mkf_b200.field_bpfd(f, t, mkf_b200.BMC_GT, out=out)
        e1.record()
        torch.cuda.synchronize(dev)
        dev_ms.append(e0.elapsed_time(e1))
        if step < streamed_steps:
            h.copy_(f)
            t0 = time.perf_counter()
            hc = mkf_b200.field_bpfd_host(h.numpy(), t, mkf_b200.BMC_GT)
            host_s.append(time.perf_counter() - t0)
            same = same and bool((hc == out.cpu().numpy().view(np.uint64)).all())
    del f, h
    torch.cuda.empty_cache()
    return {
        "workload": "2048 x 2048 x 1536 FP32 plane-wave series, 256 waves, thresholds {-0.5, 0, 0.5}",
        "steps_device_resident": steps,
        "steps_streamed": streamed_steps,
        "device_resident_ms_per_step": float(np.mean(dev_ms)),
        "device_resident_ms_per_step_min_max": [float(np.min(dev_ms)), float(np.max(dev_ms))],
        "device_resident_gvoxel_per_s": vox / (np.mean(dev_ms) * 1e-3) * 1e-9,
        "device_resident_gb_per_s": vox * 4 / (np.mean(dev_ms) * 1e-3) * 1e-9,
        "streamed_s_per_step": float(np.mean(host_s)),
        "streamed_gvoxel_per_s": vox / np.mean(host_s) * 1e-9,
        "streamed_h2d_gb_per_s": vox * 4 / np.mean(host_s) * 1e-9,
        "device_equals_streamed": same,
    }


# ---------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 50 ms in the background."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.rows = []
        self.proc = None
        self.gpu_id = gpu_id
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.gpu_id, "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return

        def reader():
            for line in self.proc.stdout:
                self.rows.append((time.time(), [c.strip() for c in line.split(",")]))

        self.thread = threading.Thread(target=reader, daemon=True)
        self.thread.start()

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)

    def summary(self, t0, t1):
        rows = [r for ts, r in self.rows if t0 <= ts <= t1 and len(r) >= 9]
        if not rows:
            after = [r for ts, r in self.rows if ts >= t0 and len(r) >= 9]
            rows = after[:3]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if num(r[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def gpu_id_of(dev_index: int) -> str:
    import torch

    try:
        p = torch.cuda.get_device_properties(dev_index)
        return "%08X:%02X:%02X.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
    except Exception:
        return str(dev_index)


def measured_hbm_peak():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per launch of the fused kernel from the committed ncu summary, if present."""
    path = os.path.join(REPO, "profiles", "thermo_tma_grf_f64_k16.md")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_launch_full:"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


# ---------------------------------------------------------------- CPU runs (reference C path)

def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_sample(f: np.ndarray, planes: int, threads: int):
    """Time the reference C path on planes+1 planes (1024 x 1024, FP64) of f, all 16 thresholds
    (one reference call per threshold, as its interface takes one). Returns (s, voxels, kind, threads)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    from oracle import Oracle, RefOracle

    nz = planes + 1
    d = (N_SIDE, N_SIDE, nz)
    slab = f[: nz * N_SIDE * N_SIDE]
    if RefOracle.available():
        ref = RefOracle()
        t0 = time.perf_counter()
        for t in THRESHOLDS:
            ref.bpfd_mt(slab, d, float(t), 4, threads)
        dt = time.perf_counter() - t0
        kind = "reference"
    else:  # the project's port of the same algorithm (single thread)
        orc = Oracle()
        t0 = time.perf_counter()
        orc.bpfd_field(np.ascontiguousarray(slab).reshape(nz, N_SIDE, N_SIDE), d, THRESHOLDS, [4] * K_THRESH)
        dt = time.perf_counter() - t0
        kind, threads = "port", 1
    return dt, planes * N_SIDE * N_SIDE, kind, threads


def calibrate_planes(f: np.ndarray, threads: int, target_s: float, max_planes: int) -> int:
    """Plane pairs per sample for about target_s seconds of reference work: a two-point fit (8 and
    32 planes) separates the per-plane cost from the fixed cost of each call's thread start-up."""
    n1, n2 = min(8, max_planes), min(32, max_planes)
    t1, _, _, _ = reference_sample(f, n1, threads)
    if n2 <= n1:
        return int(max(2, min(max_planes, n1 * target_s / max(t1, 1e-4))))
    t2, _, _, _ = reference_sample(f, n2, threads)
    per_plane = max((t2 - t1) / (n2 - n1), 1e-6)
    fixed = max(t1 - n1 * per_plane, 0.0)
    return int(max(2, min(max_planes, (target_s - fixed) / per_plane)))


def cpu_baseline(f: np.ndarray, counts: np.ndarray | None = None, target_s: float = 10.0):
    """The reference C path on this host's cores over the whole benchmark field (all 1023 plane
    pairs, one reference call per threshold, each split into z-slabs over every host thread), its
    counts compared with `counts` (the GPU's, uint64 [16, 256]) bin by bin as the reference's own
    test compares its CPU and GPU distributions (mkfTest.c:64-85); plus the reference's
    single-thread entry point exactly as written (mkfAccGetBPFDSimple, mkfACC.c:206-239) on a
    16-plane slab. Without the reference build, the project's port on a calibrated slab."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    from oracle import RefOracle

    threads = cpu_threads()
    if not RefOracle.available():
        planes = calibrate_planes(f, threads, target_s, N_SIDE - 1)
        dt, vox, kind, thr = reference_sample(f, planes, threads)
        return {"value": vox / dt * 1e-9, "unit": "Gvoxel/s", "cores": thr, "kind": kind,
                "sample": f"{planes} plane pairs of the 1024^3 FP64 benchmark field, 16 thresholds, {dt:.2f} s"}, None
    ref = RefOracle()
    d = (N_SIDE, N_SIDE, N_SIDE)
    t0 = time.perf_counter()
    want = np.stack([ref.bpfd_mt(f, d, float(t), 4, threads) for t in THRESHOLDS])
    dt = time.perf_counter() - t0
    res = {"value": N_SIDE ** 3 / dt * 1e-9, "unit": "Gvoxel/s", "cores": threads, "kind": "reference",
           "sample": f"the whole 1024^3 FP64 benchmark field (1023 plane pairs), 16 thresholds (16 reference "
                     f"calls, z-slabs over {threads} threads), {dt:.2f} s"}
    if counts is not None:
        res["counts_equal_gpu"] = bool((want == counts).all())
    # single thread, as written: one mkfAccGetBPFDSimple call per threshold on 16 plane pairs
    nz = 17
    slab = np.ascontiguousarray(f[: nz * N_SIDE * N_SIDE]).reshape(nz, N_SIDE, N_SIDE)
    t0 = time.perf_counter()
    one = np.stack([ref.bpfd_simple(slab, (N_SIDE, N_SIDE, nz), float(t), 4) for t in THRESHOLDS])
    dt1 = time.perf_counter() - t0
    mt = np.stack([ref.bpfd_mt(slab.ravel(), (N_SIDE, N_SIDE, nz), float(t), 4, threads) for t in THRESHOLDS])
    res["single_thread"] = {"value": (nz - 1) * N_SIDE * N_SIDE / dt1 * 1e-9, "unit": "Gvoxel/s", "cores": 1,
                            "entry_point": "mkfAccGetBPFDSimple (mkfACC.c:206-239)",
                            "sample": f"16 plane pairs x 1024 x 1024 of the benchmark field, 16 thresholds, {dt1:.2f} s",
                            "counts_equal_multithreaded": bool((one == mt).all())}
    return res, want


def ball256_torch(device, seed=11):
    """The plain method's workload: 256^3 FP32, 100 - |x - c| (c = 127.5 on each axis) plus
    U[-0.5, 0.5) noise from a fixed seed; threshold 0, relation '>'."""
    import torch

    n, c = 256, 127.5
    ax = torch.arange(n, dtype=torch.float64, device=device) - c
    f = 100.0 - torch.sqrt(ax.view(-1, 1, 1) ** 2 + ax.view(1, -1, 1) ** 2 + ax.view(1, 1, -1) ** 2)
    g = torch.Generator(device=device).manual_seed(seed)
    f += torch.rand((n, n, n), dtype=torch.float64, device=device, generator=g) - 0.5
    return f.float().contiguous()


def reference_cuda(args):
    """The reference's own CUDA path (binMapCUDA + mkfCUDAGetBPFD with the FAST profile, one call
    pair per threshold as its one-threshold interface requires), compiled unmodified from its
    sources for sm_100a, on the benchmark field resident in HBM and on the 256^3 FP32 ball.
    Device-timed with CUDA events around each step; the reference synchronises after each of its
    stages itself (utilCUDA.hpp:21-60), which is part of its cost."""
    try:
        import torch

        if not torch.cuda.is_available():
            return {"unavailable": "no CUDA device"}
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        from oracle import RefCuda
    except Exception as e:  # noqa: BLE001 - reported, not fatal to the CPU arm
        return {"unavailable": f"{type(e).__name__}: {e}"}
    if not RefCuda.available():
        return {"unavailable": "reference CUDA build (oracle/_ref/libmkfrefcuda.so) missing"}
    ref = RefCuda()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)

    flush = torch.empty(64 << 20, dtype=torch.int32, device=dev)  # 256 MB > 126 MB L2

    def timed(f, thresholds, workload, flush_l2):
        Z, Y, X = f.shape
        d = (X, Y, Z)
        pbm = torch.empty(ref.pbm_words(d), dtype=torch.int32, device=dev)
        counts = torch.zeros((len(thresholds), 256), dtype=torch.int64, device=dev)

        def one():
            counts.zero_()
            return ref.bpfd(counts.data_ptr(), pbm.data_ptr(), f.data_ptr(), f.element_size(), d, thresholds, ">")

        for _ in range(max(args.warmup, 1)):
            one()
        torch.cuda.synchronize(dev)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        t_map = t_bpfd = 0.0
        for e0, e1 in ev:
            if flush_l2:
                flush.zero_()
            e0.record(stream)
            a, b = one()
            e1.record(stream)
            t_map += a
            t_bpfd += b
        torch.cuda.synchronize(dev)
        ms = sum(e0.elapsed_time(e1) for e0, e1 in ev) / args.steps
        return {"workload": workload, "ms_per_step": ms, "gvoxel_per_s": X * Y * Z / ms * 1e-6,
                "map_ms_per_step": t_map / args.steps, "bpfd_ms_per_step": t_bpfd / args.steps,
                "launches_per_step": 2 * len(thresholds),
                "l2": "flushed before each step" if flush_l2 else "input larger than L2 (no flush)"}

    out = {"build": "reference binMapCUDA.cu, mkfCUDA.cu, ctUtil.cu, gridUtil.cu (+ binMapUtil.c, encoding.c, "
                    "geomSVU.c) compiled unmodified, nvcc -gencode arch=compute_100a,code=sm_100a -O3",
           "thresholds": "rounded to float by the reference's interface (binMapUtil.c:37)"}
    f = grf_torch(N_SIDE, N_SIDE, N_SIDE, SEED, dev)
    out[WORKLOAD] = timed(f, THRESHOLDS, f"{N_SIDE}^3 FP64 GRF, {K_THRESH} thresholds (16 call pairs)", False)
    del f
    f = ball256_torch(dev)
    out["ball256_f32_k1"] = timed(f, [0.0], "256^3 FP32 ball, threshold 0 (1 call pair)", True)
    del f, flush
    torch.cuda.empty_cache()
    return out


def run_reference(args, rank, world):
    if rank != 0:
        return
    threads = cpu_threads()
    max_planes = 128
    f = grf_numpy(max_planes + 1, N_SIDE, N_SIDE, SEED)  # a slab of the same kind of field (1 GB)
    planes = calibrate_planes(f, threads, 0.5, max_planes)  # about 0.5 s of reference work per step
    for _ in range(args.warmup):
        reference_sample(f, planes, threads)
    times = []
    for _ in range(args.steps):
        dt, vox, kind, thr = reference_sample(f, planes, threads)
        times.append(dt)
    total = sum(times)
    value = args.steps * vox / total * 1e-9
    line = {
        "impl": "reference", "metric": "Gvoxel/s per field (16 thresholds)", "value": value, "unit": "Gvoxel/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "field": [N_SIDE, N_SIDE, N_SIDE], "thresholds": K_THRESH, "relation": ">",
                   "step": f"bounded sample: {planes} plane pairs x 1024 x 1024 per step"},
        "cpu_baseline": {"value": value, "unit": "Gvoxel/s", "cores": thr, "kind": kind,
                         "sample": f"{planes} plane pairs x 1024 x 1024 FP64 GRF slab per step, 16 thresholds"},
        "e2e": {"value": value, "unit": "Gvoxel/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_secondary:
        line["reference_cuda"] = reference_cuda(args)
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU run

def run_mkf(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    import mkf_b200
    from mkf_b200 import shard

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    mkf_b200.lib()
    # this rank's z-slab of a field of world x 1024 cell planes: 1024 cell planes plus one halo
    # plane (weak scaling; each slab is its own seeded GRF, generated on this rank's GPU)
    z0, z1 = shard.slab_planes(world * N_SIDE + 1, world, rank) if world > 1 else (0, N_SIDE)
    nz = z1 - z0
    f = grf_torch(nz, N_SIDE, N_SIDE, SEED + rank, dev)
    vox = N_SIDE ** 3  # voxels of the field (or of this rank's slab) per step
    stream = torch.cuda.current_stream(dev)
    out = torch.zeros((K_THRESH, 256), dtype=torch.int64, device=dev)
    meas = torch.empty((K_THRESH, 4), dtype=torch.float64, device=dev)
    ev_k = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]

    def step(i=None):
        def counter(slab, thresholds, mask, o):  # the counting kernel, bracketed by CUDA events
            if i is not None:
                ev_k[i][0].record(stream)
            mkf_b200.field_bpfd(slab, thresholds, mask, out=o, accumulate=True, stream=stream)
            if i is not None:
                ev_k[i][1].record(stream)

        # zero the counts, count this rank's slab, all-reduce the counts over the ranks (N > 1)
        shard.sharded_field_bpfd(f, THRESHOLDS, mkf_b200.BMC_GT, out=out, stream=stream, counter=counter)
        mkf_b200._lib.check(mkf_b200.lib().mkfMeasuresF64Dev(meas.data_ptr(), out.data_ptr(), K_THRESH,
                                                             stream.cuda_stream), "mkfMeasuresF64Dev")

    # slab depth measured once for this kind of field (outside the timed region)
    mkf_b200.tune(f, THRESHOLDS, mkf_b200.BMC_GT, stream=stream)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(gpu_id_of(local_rank))
    sampler.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    w0 = time.time()
    e0.record(stream)
    for i in range(args.steps):
        step(i)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    w1 = time.time()
    if world > 1:
        dist.barrier()
    time.sleep(0.1)
    sampler.stop()
    ms = e0.elapsed_time(e1)
    kern_ms = float(np.mean([a.elapsed_time(b) for a, b in ev_k]))
    # the timed kernel's counts against a different kernel (one threshold at a time, word-parallel)
    # (one GPU: with several, `out` holds the all-reduced counts of every rank's slab)
    checked = None if world > 1 else all(
        bool(torch.equal(out[k:k + 1], mkf_b200.field_bpfd(f, THRESHOLDS[k:k + 1], mkf_b200.BMC_GT)))
        for k in (0, K_THRESH // 2, K_THRESH - 1))
    t = torch.tensor([ms, kern_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms, kern_ms = float(t[0]), float(t[1])
    value = world * vox * args.steps / (ms * 1e-3) * 1e-9
    clocks = sampler.summary(w0, w1)

    # end to end through the host-buffer entry point
    fh = torch.empty(f.shape, dtype=f.dtype, pin_memory=True)
    fh.copy_(f)
    fh_np = fh.numpy()
    del f
    torch.cuda.empty_cache()
    mkf_b200.field_bpfd_host(fh_np, THRESHOLDS, mkf_b200.BMC_GT)  # warm-up (staging buffers)
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        h = mkf_b200.field_bpfd_host(fh_np, THRESHOLDS, mkf_b200.BMC_GT)
        if world > 1:
            ht = torch.from_numpy(h.view(np.int64)).to(dev)
            dist.all_reduce(ht)
            h = ht.cpu().numpy()
        mkf_b200.measures(h)
    e2e_s = (time.perf_counter() - t0) / args.e2e_steps
    tt = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    e2e_s = float(tt[0])
    e2e = {"value": world * vox / e2e_s * 1e-9, "unit": "Gvoxel/s", "h2d_bytes_per_step": int(fh.numel() * 8),
           "d2h_bytes_per_step": K_THRESH * 256 * 8}

    if rank != 0:
        return
    peak, peak_src = measured_hbm_peak()
    alg_bytes = vox * 8 + K_THRESH * 256 * 8
    achieved = alg_bytes / (kern_ms * 1e-3) * 1e-9
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": peak_src, "traffic": profiled_traffic(), "kernel_ms": kern_ms,
            "algorithmic_bytes": alg_bytes}
    line = {
        "metric": "Gvoxel/s per field (16 thresholds)", "value": value, "unit": "Gvoxel/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Gaussian random field, sigma 4, generated on the GPU)",
        "config": {"workload": WORKLOAD, "field": [N_SIDE, N_SIDE, N_SIDE], "thresholds": K_THRESH,
                   "threshold_range": [-2.0, 2.0], "relation": ">",
                   "parallelism": "replicas" if world == 1 else f"z-slab shards x{world} + NCCL all-reduce of counts",
                   "l2": "inputs 8.6 GB per step > 126 MB L2 (no flush)"},
        "roofline": roof,
        "e2e": e2e,
        "gpu_launches": 2 * args.steps,
        "counts_checked_against_word_kernel": checked,
        "clocks": clocks,
    }
    if world == 1 and not args.no_cpu_baseline:
        got = out.cpu().numpy().view(np.uint64)
        cb, _want = cpu_baseline(fh_np.reshape(-1), got)
        if "counts_equal_gpu" in cb:
            line["counts_equal_reference"] = cb.pop("counts_equal_gpu")
        line["cpu_baseline"] = cb
    if world == 1 and not args.no_secondary:
        del fh, fh_np
        line["plain"] = run_plain_workload(dev)
        line["batched"] = run_batch_workload(dev)
        line["serving"] = run_serving_workload(dev)
        line["insitu"] = run_insitu_workload(dev)
    print(json.dumps(line), flush=True)
    if line.get("counts_equal_reference") is False:
        raise SystemExit("the timed counts differ from the reference C path's")


def run_profile_case(args):
    """A small case for a profiler: 3 untimed launches, then --reps launches timed with CUDA
    events; prints one JSON line (not a benchmark result)."""
    import torch

    import mkf_b200

    dev = torch.device("cuda:0")
    mkf_b200.lib()
    if args.profile == "field":
        n = args.side
        f = grf_torch(n, n, n, 1, dev)
        f = f if args.dtype == "f64" else f.float().contiguous()
        t = (np.linspace(-2.0, 2.0, int(args.thresholds)) if "," not in args.thresholds and "." not in args.thresholds
             else np.array([float(v) for v in args.thresholds.split(",")]))
        out = torch.zeros((len(t), 256), dtype=torch.int64, device=dev)

        def launch():
            mkf_b200.field_bpfd(f, t, mkf_b200.BMC_GT, out=out)

        vox, nbytes, what = f.numel(), f.numel() * f.element_size(), f"{n}^3 {args.dtype} GRF, {len(t)} thresholds"
    elif args.profile == "planewave":
        f = torch.empty((args.side, 1024, 1024), dtype=torch.float32, device=dev)
        plane_wave_field(f, 256, SEED + 6, 0)
        t = [-0.5, 0.0, 0.5]
        out = torch.zeros((3, 256), dtype=torch.int64, device=dev)

        def launch():
            mkf_b200.field_bpfd(f, t, mkf_b200.BMC_GT, out=out)

        vox, nbytes, what = f.numel(), f.numel() * 4, f"1024 x 1024 x {args.side} FP32 plane waves, 3 thresholds"
    elif args.profile == "dropin":
        f = ball256_torch(dev)
        pbm0, org0, _ = mkf_b200.bin_map_cuda(f, ">", 0.0)
        counts = torch.zeros(256, dtype=torch.int64, device=dev)

        def launch():
            pbm, org, _ = mkf_b200.bin_map_cuda(f, ">", 0.0, out=pbm0)
            mkf_b200.get_bpfd(pbm, org, out=counts)

        vox, nbytes, what = f.numel(), f.numel() * 4, "256^3 FP32 ball, threshold 0, drop-in pair"
    else:
        fields = ball_fields(args.fields, 77, dev)
        plan = mkf_b200.BatchPlan(fields, [[0.0]] * len(fields))  # tunes the slab depth at creation

        def launch():
            plan.launch()

        vox = sum(x.numel() for x in fields)
        nbytes, what = vox * 4, f"{len(fields)} FP32 ball fields, threshold 0"
    for _ in range(3):
        launch()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.reps):
        launch()
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / args.reps
    print(json.dumps({"profile_case": what, "ms_per_launch": ms, "gvoxel_per_s": vox / ms * 1e-6,
                      "field_gb_per_s": nbytes / ms * 1e-6}), flush=True)
    if args.profile == "batch":
        plan.close()


def main():
    args = parse()
    if args.profile:
        run_profile_case(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_mkf(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
