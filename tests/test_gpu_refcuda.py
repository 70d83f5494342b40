"""Parity against the reference's own CUDA path (binMapCUDA + mkfCUDAGetBPFD, mkfCUDA.cu:12-61,
binMapCUDA.cu:144-264) compiled unmodified for sm_100a, run on the same device tensors as this
library. The reference takes one threshold per call and rounds it to float (binMapUtil.c:37), so
this library is given the same float-rounded thresholds as doubles; the counts must then agree
bit for bit. The reference path is defined only for one planar field with X a multiple of 32 (a
row's words 0 .. X/32 - 1 are read, bpfdCUDA.cuh:92-118), so every case here has such an X."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref_cuda():
    from oracle import RefCuda

    if not RefCuda.available():
        pytest.skip("reference CUDA library (oracle/_ref) not built on this machine")
    return RefCuda()


def _grf(shape_zyx, seed, dev, dtype):
    import bench

    return bench.grf_torch(*shape_zyx, seed, dev).to(dtype).contiguous()


def _ours(mkf, f, t, rel_mask):
    return mkf.field_bpfd(f, t, rel_mask).cpu().numpy().view(np.uint64)


def test_ball256_fp32_equals_reference_cuda(mkf, ref_cuda, cuda):
    """The plain-method case: 256^3 FP32 ball (100 - |x - c|, c = 127.5, U[-0.5, 0.5) noise), f > 0."""
    import torch

    n = 256
    c = 127.5
    ax = torch.arange(n, dtype=torch.float64, device=cuda) - c
    f = 100.0 - torch.sqrt(ax.view(-1, 1, 1) ** 2 + ax.view(1, -1, 1) ** 2 + ax.view(1, 1, -1) ** 2)
    g = torch.Generator(device=cuda).manual_seed(11)
    f = (f + torch.rand((n, n, n), dtype=torch.float64, device=cuda, generator=g) - 0.5).float().contiguous()
    want = ref_cuda.bpfd_torch(f, [0.0], ">")
    assert int(want.sum()) == 255 ** 3
    assert (_ours(mkf, f, [0.0], mkf.BMC_GT) == want).all()


@pytest.mark.parametrize("dtype_name", ["f64", "f32"])
def test_grf_sixteen_thresholds_equal_reference_cuda(mkf, ref_cuda, cuda, dtype_name):
    """The benchmark's kind of field (Gaussian random field, sigma 4) at 96 x 80 x 256, the 16
    thresholds linspace(-2, 2, 16) rounded to float: the reference's 16 call pairs against one
    call of this library (rank-table kernel)."""
    import torch

    dtype = torch.float64 if dtype_name == "f64" else torch.float32
    f = _grf((96, 80, 256), 5, cuda, dtype)
    t = np.linspace(-2.0, 2.0, 16).astype(np.float32).astype(np.float64)
    want = ref_cuda.bpfd_torch(f, t, ">")
    assert (want.sum(axis=1) == 95 * 79 * 255).all()
    assert (_ours(mkf, f, t, mkf.BMC_GT) == want).all()


@pytest.mark.parametrize("rel,mask", [("<=", 3), ("!=", 5), ("=", 2), (">=", 6)])
def test_relations_equal_reference_cuda(mkf, ref_cuda, cuda, rel, mask):
    """Every relation the reference's string form can state (binMapUtil.c:37-58), on an FP32 field
    quantised to quarter steps so that equality with the thresholds occurs; 3 thresholds (word
    kernel) and 7 (rank-table kernel)."""
    import torch

    f = (torch.round(_grf((40, 64, 128), 9, cuda, torch.float32) * 4) / 4).contiguous()
    for t in ([-0.5, 0.0, 0.75], [-1.5, -1.0, -0.25, 0.0, 0.25, 1.0, 1.5]):
        want = ref_cuda.bpfd_torch(f, t, rel)
        assert (_ours(mkf, f, t, mask) == want).all(), (rel, t)
