"""Parity cases for the workloads other than the benchmark one: the 256^3 FP32 ball of the plain
method (checked against the reference's own C path, exactly) and the plane-wave in-situ series
(checked through size-independent properties and an oracle sub-block, device-resident and streamed
from pinned host memory)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ball256(seed=11):
    n = 256
    c = 127.5
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    f = 100.0 - np.sqrt((x - c) ** 2 + (y - c) ** 2 + (z - c) ** 2)
    f += np.random.default_rng(seed).uniform(-0.5, 0.5, size=f.shape)
    return f.astype(np.float32)


def test_plain_method_ball_equals_reference(mkf, oracle, ref_oracle, cuda):
    """256^3 FP32 ball, f > 0: the drop-in pair and the fused call against the reference C path on
    the same values (the reference reads FP64; float -> double is exact and the threshold 0 is a
    float), and the measures of the fused counts against the oracle's."""
    import torch

    f = _ball256()
    d = (256, 256, 256)
    want = ref_oracle.bpfd_mt(ref_oracle.padded(f), d, 0.0, mkf.BMC_GT, os.cpu_count() or 1)
    assert int(want.sum()) == 255 ** 3
    fd = torch.from_numpy(f).to(cuda)
    pbm, org, _ = mkf.bin_map_cuda(fd, ">", 0.0)
    assert (mkf.get_bpfd_host(pbm, org) == want).all()
    fused = mkf.field_bpfd(fd, [0.0], mkf.BMC_GT).cpu().numpy().view(np.uint64)
    assert (fused[0] == want).all()
    r = mkf.measures(fused)[0]
    assert (r == oracle.measures(want)).all()


def _plane_waves(shape_zyx, n_waves, seed, dev, step):
    """Sum of n_waves plane waves (unit-norm random directions, |k| uniform in [0.05, 0.1]
    rad/voxel, phases from the seed, each advanced by its own rotation per step), scaled to unit
    variance; plane z is Re((A_y * a_z) @ A_x^T) with A_x[x, w] = exp(i k_x,w x)."""
    import torch

    rng = np.random.default_rng(seed)
    d = rng.standard_normal((n_waves, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    kv = d * rng.uniform(0.05, 0.1, size=n_waves)[:, None]
    ph = rng.uniform(0, 2 * np.pi, size=n_waves) + step * rng.uniform(-0.3, 0.3, size=n_waves)
    Z, Y, X = shape_zyx
    cx = torch.tensor(kv[:, 0], dtype=torch.float64, device=dev)
    cy = torch.tensor(kv[:, 1], dtype=torch.float64, device=dev)
    ax = torch.exp(1j * torch.arange(X, dtype=torch.float64, device=dev)[:, None] * cx[None, :]).to(torch.complex64)
    ay = torch.exp(1j * torch.arange(Y, dtype=torch.float64, device=dev)[:, None] * cy[None, :]).to(torch.complex64)
    f = torch.empty((Z, Y, X), dtype=torch.float32, device=dev)
    for z in range(Z):
        az = torch.exp(1j * torch.tensor(kv[:, 2] * z + ph, dtype=torch.float64, device=dev)).to(torch.complex64)
        f[z] = ((ay * az[None, :]) @ ax.T).real * float(np.sqrt(2.0 / n_waves))
    return f


def test_insitu_plane_wave_series(mkf, oracle, cuda):
    """2048 x 2048 planes of the plane-wave series (a 24-plane slab of the 1536), thresholds
    {-0.5, 0, 0.5}, two time steps: the device-resident pass, the pass streamed from pinned host
    memory and one single-threshold call per threshold agree exactly; every distribution sums to
    the cell count; a 12 x 80 x 100 block matches the oracle."""
    import torch

    t = [-0.5, 0.0, 0.5]
    shape = (24, 2048, 2048)
    cells = 23 * 2047 * 2047
    for step in range(2):
        f = _plane_waves(shape, 256, 21, cuda, step)
        dev = mkf.field_bpfd(f, t, mkf.BMC_GT).cpu().numpy().view(np.uint64)
        assert (dev.sum(axis=1) == cells).all()
        h = torch.empty(shape, dtype=torch.float32, pin_memory=True)
        h.copy_(f)
        host = mkf.field_bpfd_host(h.numpy(), t, mkf.BMC_GT)
        assert (host == dev).all()
        for k, tv in enumerate(t):
            one = mkf.field_bpfd(f, [tv], mkf.BMC_GT).cpu().numpy().view(np.uint64)
            assert (one[0] == dev[k]).all()
        blk = f[6:18, 1000:1080, 500:600].cpu().numpy()
        got = mkf.field_bpfd(f[6:18, 1000:1080, 500:600], t, mkf.BMC_GT).cpu().numpy().view(np.uint64)
        assert (got == oracle.bpfd_field(np.ascontiguousarray(blk), (100, 80, 12), t, mkf.BMC_GT)).all()
        del f, h
