"""Parity of the CUDA library (through its C ABI) with the oracle and the reference's golden
vectors. Integer outputs must be bit-exact; the double measures must equal the host's exactly.
Needs a B200 (`-m gpu`)."""
import os
import sys

import numpy as np
import pytest

from oracle import bpfd_numpy, layout

pytestmark = pytest.mark.gpu


def to_dev(a, cuda):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def u64(t):
    return t.cpu().numpy().view(np.uint64)


def valid_bits_mask(X, Y, Z):
    row, _ = layout((X, Y, Z))
    m = np.zeros(row, np.uint32)
    for w in range(row):
        nb = min(32, X - 32 * w)
        m[w] = np.uint32((1 << nb) - 1) if nb < 32 else np.uint32(0xFFFFFFFF)
    return np.tile(m, Y * Z)


# ---------------------------------------------------------------- fused (K thresholds, one read)

def test_fused_golden_cases(mkf, golden, oracle, cuda):
    for key in [str(n) for n in golden["names"] if not str(n).startswith("short_")]:
        f = golden[key + "/field"]
        t, m = golden[key + "/t"], golden[key + "/m"]
        got = u64(mkf.field_bpfd(to_dev(f, cuda), t, m))
        assert (got == golden[key + "/bpfd"]).all(), key


def test_fused_short_rows(mkf, golden, oracle, cuda):
    for key in [str(n) for n in golden["names"] if str(n).startswith("short_")]:
        f = golden[key + "/field"]
        Z, Y, X = f.shape
        got = u64(mkf.field_bpfd(to_dev(f, cuda), [0.0], 4))[0]
        assert (got == oracle.bpfd_field(f, (X, Y, Z), 0.0, 4)[0]).all(), key


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("seed", range(5))
def test_fused_random_shapes(mkf, oracle, cuda, dtype, seed):
    rng = np.random.default_rng(1000 + seed)
    for _ in range(5):
        X = int(rng.choice([1, 2, 3, 17, 31, 32, 33, 63, 64, 65, 100, 129]))
        Y = int(rng.integers(1, 40))
        Z = int(rng.integers(1, 80))
        f = (rng.standard_normal((Z, Y, X)) * 1.5).astype(dtype)
        K = int(rng.integers(1, 33))
        t = np.sort(rng.standard_normal(K)) if seed % 2 else rng.standard_normal(K)
        mask = int(rng.choice([4, 6, 1, 3]))
        got = u64(mkf.field_bpfd(to_dev(f, cuda), t, mask))
        want = oracle.bpfd_field(f, (X, Y, Z), t, mask)
        assert (got == want).all(), (X, Y, Z, K, mask)


@pytest.mark.parametrize("seed", range(4))
def test_fused_mixed_relations_and_ties(mkf, oracle, cuda, seed):
    rng = np.random.default_rng(2000 + seed)
    X, Y, Z = 45, 23, 19
    f = rng.integers(-3, 4, size=(Z, Y, X)).astype(np.float64) * 0.5
    K = 12
    t = rng.integers(-3, 4, size=K).astype(np.float64) * 0.5
    m = rng.integers(0, 8, size=K).astype(np.uint32)
    got = u64(mkf.field_bpfd(to_dev(f, cuda), t, m))
    assert (got == oracle.bpfd_field(f, (X, Y, Z), t, m)).all()
    f32 = f.astype(np.float32)
    got = u64(mkf.field_bpfd(to_dev(f32, cuda), t, m))
    assert (got == oracle.bpfd_field(f32, (X, Y, Z), t, m)).all()


def test_fused_special_values(mkf, oracle, cuda):
    rng = np.random.default_rng(7)
    f = rng.standard_normal((9, 13, 70))
    flat = f.ravel()
    idx = rng.choice(flat.size, 400, replace=False)
    flat[idx[:80]] = np.nan
    flat[idx[80:160]] = np.inf
    flat[idx[160:240]] = -np.inf
    flat[idx[240:320]] = 0.0
    flat[idx[320:]] = -0.0
    Z, Y, X = f.shape
    ts = [0.0, -0.0, np.inf, -np.inf, np.nan, 0.5, 1e300, -1e-300]
    for mask in range(8):
        got = u64(mkf.field_bpfd(to_dev(f, cuda), ts, mask))
        assert (got == oracle.bpfd_field(f, (X, Y, Z), ts, [mask] * len(ts))).all(), mask
        f32 = f.astype(np.float32)
        got = u64(mkf.field_bpfd(to_dev(f32, cuda), ts, mask))
        assert (got == oracle.bpfd_field(f32, (X, Y, Z), ts, [mask] * len(ts))).all(), mask


def test_fused_fp32_thresholds_not_rounded(mkf, oracle, cuda):
    """A FP32 field compared with a double threshold that no float represents: the result is
    that of the exact comparison (as if the element were promoted to double)."""
    f = np.full((4, 4, 40), np.float32(0.1), np.float32)
    f[:, :, ::3] = np.nextafter(np.float32(0.1), np.float32(1))
    t = [0.1, float(np.float32(0.1)), 0.1 + 1e-12]
    for mask in (1, 2, 3, 4, 5, 6):
        got = u64(mkf.field_bpfd(to_dev(f, cuda), t, mask))
        assert (got == oracle.bpfd_field(f, (40, 4, 4), t, [mask] * 3)).all(), mask


def test_fused_strided_view(mkf, oracle, cuda):
    import torch

    rng = np.random.default_rng(11)
    big = rng.standard_normal((30, 40, 50))
    v = to_dev(big, cuda)[2:27:2, 5:35, 3:47]  # non-contiguous view (Z step 2)
    sub = np.ascontiguousarray(big[2:27:2, 5:35, 3:47])
    Z, Y, X = sub.shape
    got = u64(mkf.field_bpfd(v, [-0.3, 0.2, 0.9], 4))
    assert (got == oracle.bpfd_field(sub, (X, Y, Z), [-0.3, 0.2, 0.9], 4)).all()
    vt = to_dev(big, cuda).permute(0, 2, 1)  # x and y swapped: x stride is not 1
    subt = np.ascontiguousarray(big.transpose(0, 2, 1))
    Z, Y, X = subt.shape
    got = u64(mkf.field_bpfd(vt, [0.1], 6))
    assert (got == oracle.bpfd_field(subt, (X, Y, Z), [0.1], 6)).all()


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_fused_one_or_two_thresholds_every_relation(mkf, oracle, cuda, dtype):
    """The word-parallel path: K = 1, 2 with every relation pair, ties, NaN. Fields narrower than
    32 in x or y take the clamped tiles; larger ones the shifted edge tiles (x and y not multiples
    of 31), strided views both."""
    rng = np.random.default_rng(71)
    for shape in [(9, 11, 64), (7, 13, 100), (5, 6, 1030), (6, 9, 33), (4, 5, 2), (3, 40, 993),
                  (5, 45, 100), (4, 64, 64), (3, 33, 32), (34, 32, 63)]:
        f = (rng.integers(-4, 5, size=shape) * 0.5).astype(dtype)
        f.ravel()[rng.choice(f.size, max(1, f.size // 50), replace=False)] = np.nan
        Z, Y, X = shape
        for m0 in range(8):
            m1 = (m0 * 5 + 3) % 8
            for t in ([0.5], [0.0, -1.0]):
                m = [m0, m1][: len(t)]
                got = u64(mkf.field_bpfd(to_dev(f, cuda), t, m))
                assert (got == oracle.bpfd_field(f, (X, Y, Z), t, m)).all(), (shape, m, t)
    big = to_dev(rng.standard_normal((12, 30, 140)).astype(dtype), cuda)
    big2 = to_dev(rng.standard_normal((10, 70, 150)).astype(dtype), cuda)
    for view in (big[1:11, 2:28, 4:132], big[:, :, ::2], big.permute(0, 2, 1),
                 big2[1:9, 3:67, 5:140], big2[:, :, ::2], big2.permute(0, 2, 1), big2.permute(2, 1, 0)):
        sub = np.ascontiguousarray(view.cpu().numpy())
        Z, Y, X = sub.shape
        for t, m in (([0.1], [4]), ([0.1, -0.2], [6, 1])):
            got = u64(mkf.field_bpfd(view, t, m))
            assert (got == oracle.bpfd_field(sub, (X, Y, Z), t, m)).all()


def test_fused_accumulate(mkf, cuda):
    rng = np.random.default_rng(3)
    f = to_dev(rng.standard_normal((20, 30, 40)), cuda)
    a = mkf.field_bpfd(f, [0.0, 0.5], 4)
    b = mkf.field_bpfd(f, [0.0, 0.5], 4, out=a.clone(), accumulate=True)
    assert (u64(b) == 2 * u64(a)).all()


# ---------------------------------------------------------------- size-independent properties at full size

def test_full_size_multi_threshold_properties(mkf, oracle, cuda):
    """1024^3 FP64, 16 thresholds in [-2, 2]: every distribution sums to the cell count; '>' and
    '<=' are complements; counting two z-slabs sharing a plane gives the full counts; a 64^3
    block matches the oracle exactly."""
    import torch

    n = 1024
    g = torch.Generator(device=cuda).manual_seed(5)
    f = torch.randn((n, n, n), dtype=torch.float64, device=cuda, generator=g)
    f = (f + f.roll(1, 0) + f.roll(1, 1) + f.roll(1, 2)) * 0.5  # some spatial correlation
    t = np.linspace(-2, 2, 16)
    h_gt = u64(mkf.field_bpfd(f, t, 4))
    cells = (n - 1) ** 3
    assert (h_gt.sum(axis=1) == cells).all()
    h_le = u64(mkf.field_bpfd(f, t, 3))
    assert (h_le == h_gt[:, ::-1]).all()
    h_a = u64(mkf.field_bpfd(f[:600], t, 4))
    h_b = u64(mkf.field_bpfd(f[599:], t, 4))
    assert (h_a + h_b == h_gt).all()
    # all-ones counts fall and all-zero counts rise with the threshold
    assert (np.diff(h_gt[:, 255].astype(np.int64)) <= 0).all()
    assert (np.diff(h_gt[:, 0].astype(np.int64)) >= 0).all()
    blk = f[100:164, 300:364, 700:764].contiguous()
    hb = u64(mkf.field_bpfd(blk, t, 4))
    assert (hb == oracle.bpfd_field(blk.cpu().numpy(), (64, 64, 64), t, 4)).all()
    # one and two thresholds (the word-parallel kernel) agree with rows of the 16-threshold pass
    assert (u64(mkf.field_bpfd(f, t[7:8], 4)) == h_gt[7:8]).all()
    assert (u64(mkf.field_bpfd(f, t[3:5], 4)) == h_gt[3:5]).all()
    assert (u64(mkf.field_bpfd(f, t[3:5], 3)) == h_le[3:5]).all()
    del f


# ---------------------------------------------------------------- drop-in: binMapCUDA + mkfCUDAGetBPFD

@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_dropin_golden(mkf, golden, cuda, dtype):
    for key in [str(n) for n in golden["names"] if not str(n).startswith("short_")]:
        f = golden[key + "/field"].astype(dtype)
        Z, Y, X = f.shape
        vm = valid_bits_mask(X, Y, Z)
        for k, (t, m) in enumerate(zip(golden[key + "/t"], golden[key + "/m"])):
            if np.isinf(t):
                continue
            rel = {1: "<", 2: "=", 3: "<=", 4: ">", 5: "!=", 6: ">=", 7: "<=>", 0: ""}[int(m)]
            pbm, org, ki = mkf.bin_map_cuda(to_dev(f, cuda), rel, float(t))
            words = pbm.cpu().numpy().view(np.uint32)[: vm.size]
            if dtype == np.float64 or key.startswith("int_"):
                assert ((words & vm) == (golden[key + "/pbm"][k] & vm)).all(), (key, k)
                assert (mkf.get_bpfd_host(pbm, org) == golden[key + "/bpfd"][k]).all(), (key, k)
            pad = words & ~vm
            assert (pad == 0).all()


@pytest.mark.parametrize("seed", range(4))
def test_dropin_random_vs_oracle(mkf, oracle, cuda, seed):
    rng = np.random.default_rng(3000 + seed)
    for _ in range(6):
        X = int(rng.choice([5, 31, 32, 33, 64, 70, 200]))
        Y, Z = int(rng.integers(2, 30)), int(rng.integers(2, 30))
        dtype = [np.float32, np.float64][seed % 2]
        f = rng.standard_normal((Z, Y, X)).astype(dtype)
        t = float(np.float32(rng.standard_normal()))
        pbm, org, _ = mkf.bin_map_cuda(to_dev(f, cuda), ">", t)
        assert (org.rowElem, org.rowPairs, org.planePairs) == (X, Y - 1, Z - 1)
        want_map = oracle.pack(f, (X, Y, Z), t, 4)
        assert (pbm.cpu().numpy().view(np.uint32)[: want_map.size] == want_map).all()
        want = oracle.bpfd_field(f, (X, Y, Z), t, 4)[0]
        assert (mkf.get_bpfd_host(pbm, org) == want).all()
        # mkfCUDAGetBPFD accumulates into the caller's device array
        acc = mkf.get_bpfd(pbm, org)
        acc = mkf.get_bpfd(pbm, org, out=acc)
        assert (u64(acc) == 2 * want).all()


def test_dropin_multi_field_sum_and_strides(mkf, oracle, cuda):
    import torch

    rng = np.random.default_rng(17)
    for dtype in (np.float32, np.float64):
        fs = [rng.standard_normal((11, 13, 45)).astype(dtype) for _ in range(3)]
        pbm, org, _ = mkf.bin_map_cuda([to_dev(a, cuda) for a in fs], ">=", 0.25)
        want = oracle.pack(fs, (45, 13, 11), 0.25, 6)
        assert (pbm.cpu().numpy().view(np.uint32)[: want.size] == want).all()
    # element strides given explicitly: a (Z, Y, X) view inside a larger array
    big = rng.standard_normal((12, 20, 70)).astype(np.float64)
    d = to_dev(big, cuda)
    view = d[1:11, 2:18, 5:60]
    sub = np.ascontiguousarray(big[1:11, 2:18, 5:60])
    pbm, org, _ = mkf.bin_map_cuda(view, ">", 0.1, strides_zyx=view.stride())
    want = oracle.pack(sub, (55, 16, 10), 0.1, 4)
    assert (pbm.cpu().numpy().view(np.uint32)[: want.size] == want).all()


def test_dropin_unit_dimensions_collapse(mkf, oracle, cuda):
    rng = np.random.default_rng(19)
    f = rng.standard_normal((40, 33, 1))  # X = 1: the map is laid out as 33 x 40 x 1
    pbm, org, _ = mkf.bin_map_cuda(to_dev(f, cuda), ">", 0.0)
    assert (org.rowElem, org.rowPairs, org.planePairs) == (33, 39, 0)
    want = oracle.pack(f.reshape(1, 40, 33), (33, 40, 1), 0.0, 4)
    assert (pbm.cpu().numpy().view(np.uint32)[: want.size] == want).all()
    assert (mkf.get_bpfd_host(pbm, org) == 0).all()


def test_dropin_auto_context(mkf, oracle, cuda):
    import ctypes as C

    rng = np.random.default_rng(23)
    X, Y, Z = 64, 20, 12
    f = rng.standard_normal((Z, Y, X)).astype(np.float32)
    L = mkf.lib()
    ctx = mkf._lib.Context()
    ctx.nField, ctx.nElem, ctx.enc, ctx.bytesElem = 1, X * Y * Z, mkf.ENC_F32, 4
    ctx.bytesF = f.nbytes
    words = L.setBMO(C.byref(ctx.bmo), (C.c_int * 3)(X, Y, Z), b"\x00")
    ctx.nU, ctx.bytesU = words, words * 4
    ctx.nZ, ctx.bytesZ = 256, 2048
    assert L.cuBuffAlloc(C.byref(ctx), 0) == 1
    C.memmove(ctx.pHF, f.ctypes.data, f.nbytes)
    bm = mkf.BinMapF64()
    L.setBinMapF64(C.byref(bm), b">", 0.0)
    assert L.mkfCUDAGetBPFDautoCtx(C.byref(ctx), (C.c_int * 3)(X, Y, Z), C.byref(bm), 0) == 1
    got_map = np.ctypeslib.as_array(C.cast(ctx.pHU, C.POINTER(C.c_uint32)), shape=(words,)).copy()
    assert (got_map == oracle.pack(f, (X, Y, Z), 0.0, 4)).all()
    # second stage: counts from the packed map already in the context
    pHF = ctx.pHF
    ctx.pHF = None
    assert L.mkfCUDAGetBPFDautoCtx(C.byref(ctx), (C.c_int * 3)(X, Y, Z), C.byref(bm), 0) == 1
    got = np.ctypeslib.as_array(C.cast(ctx.pHZ, C.POINTER(C.c_uint64)), shape=(256,)).copy()
    assert (got == oracle.bpfd_field(f, (X, Y, Z), 0.0, 4)[0]).all()
    ctx.pHF = pHF
    assert L.cuBuffRelease(C.byref(ctx)) == 1
    L.mkfCUDACleanup(1)
    L.binMapCUDACleanup()


# ---------------------------------------------------------------- host path, batch, measures

def test_host_field_path(mkf, oracle, cuda):
    rng = np.random.default_rng(29)
    # (40, 1024, 2048) FP32 has 8 MB planes, so the field is staged in two slabs
    for dtype, shape in [(np.float32, (300, 90, 101)), (np.float64, (5, 7, 33)), (np.float64, (1, 7, 33)),
                         (np.float32, (40, 1024, 2048))]:
        f = rng.standard_normal(shape).astype(dtype)
        Z, Y, X = shape
        t = [-1.0, 0.0, 0.7]
        got = mkf.field_bpfd_host(f, t, 4)
        dev = u64(mkf.field_bpfd(to_dev(f, cuda), t, 4))
        assert (got == dev).all()
        if f.size < 100000:
            assert (got == oracle.bpfd_field(f, (X, Y, Z), t, 4)).all()


def test_batch_equals_per_field(mkf, cuda):
    rng = np.random.default_rng(31)
    fields, ts = [], []
    for _ in range(9):
        shape = tuple(int(v) for v in rng.integers(17, 60, size=3))
        dtype = (np.float32, np.float64)[int(rng.integers(0, 2))]
        fields.append(to_dev(rng.standard_normal(shape).astype(dtype), cuda))
        ts.append(np.sort(rng.standard_normal(int(rng.integers(1, 9)))))
    got = u64(mkf.batch_bpfd(fields, ts))
    row = 0
    for f, t in zip(fields, ts):
        want = u64(mkf.field_bpfd(f, t, 4))
        assert (got[row:row + len(t)] == want).all()
        row += len(t)


def test_batch_plan_mixed_fields_and_graph(mkf, oracle, cuda):
    """A batch with FP32/FP64 fields, every relation, constant maps, NaN thresholds and a strided
    view; plan launches, graph replays, and a replay after the fields' contents change."""
    import torch

    rng = np.random.default_rng(37)
    fields, ts, ms = [], [], []
    for i in range(14):
        shape = (int(rng.integers(2, 40)), int(rng.integers(2, 40)), int(rng.choice([17, 31, 32, 33, 64, 90])))
        dtype = (np.float32, np.float64)[i % 2]
        fields.append(to_dev((rng.standard_normal(shape) * 1.5).astype(dtype), cuda))
        K = int(rng.integers(1, 9))
        t = rng.standard_normal(K)
        if i % 4 == 3:
            m = rng.integers(0, 8, size=K).astype(np.uint32)  # mixed relations: the field's own pass
            t[0] = np.nan
        else:
            m = int(rng.choice([1, 3, 4, 6]))
        ts.append(t)
        ms.append(m)
    big = to_dev(rng.standard_normal((20, 30, 50)), cuda)
    fields.append(big[2:18, 3:27, 5:45])  # strided view
    ts.append(np.array([0.2, -0.4]))
    ms.append(4)

    def want():
        return [oracle.bpfd_field(np.ascontiguousarray(f.cpu().numpy()), tuple(f.shape[::-1]), t,
                                  m if np.ndim(m) else [m] * len(t))
                for f, t, m in zip(fields, ts, ms)]

    plan = mkf.BatchPlan(fields, ts, ms)
    for launch in (plan.launch, plan.launch, plan.launch_graph, plan.launch_graph):
        got = u64(launch())
        row = 0
        for w in want():
            assert (got[row:row + len(w)] == w).all()
            row += len(w)
    for f in fields:
        f.mul_(-1.0)  # new contents, same buffers
    got = u64(plan.launch_graph())
    row = 0
    for w in want():
        assert (got[row:row + len(w)] == w).all()
        row += len(w)
    plan.close()


def test_device_measures_equal_host(mkf, golden, cuda):
    import torch

    hs = np.concatenate([golden[str(k) + "/bpfd"] for k in golden["names"] if not str(k).startswith("short_")])
    dev = mkf.measures_dev(torch.from_numpy(hs.view(np.int64)).to(cuda)).cpu().numpy()
    host = mkf.measures(hs)
    assert (dev == host).all()


# ---------------------------------------------------------------- z-slab shards (multi-GPU form, one GPU)

def test_slab_shards_sum_to_whole_field(mkf, oracle, cuda):
    """The per-rank work of the sharded form: slabs cut by slab_planes, counted one after another
    on one GPU with no process group, sum to the whole field's counts."""
    from mkf_b200.shard import sharded_field_bpfd, slab_planes

    rng = np.random.default_rng(12)
    f = rng.standard_normal((50, 70, 90))
    fd = to_dev(f, cuda)
    t = [-0.5, 0.0, 0.7]
    want = oracle.bpfd_field(f, (90, 70, 50), t, 4)
    for world in (2, 3, 4):
        tot = np.zeros_like(want)
        for r in range(world):
            z0, z1 = slab_planes(50, world, r)
            tot += u64(sharded_field_bpfd(fd[z0:z1], t, 4))
        assert (tot == want).all(), world


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_thresholds_sharing_rank_table_buckets(mkf, oracle, cuda, dtype):
    """Thresholds closer than a rank-table bucket (2 to 4 per bucket, duplicates; 5 per bucket
    takes the general kernel), elements on and between them, single-field and batched."""
    import torch

    rng = np.random.default_rng(17)
    sets = [
        [0.5, 0.5001, 0.52, 0.6, -1.0, 2.0],               # four in [0.5, 0.625)
        [1.0, 1.0, 1.1, 1.2, 3.0],                          # a duplicate and three in one bucket
        [0.25, 0.26, 0.27, 0.28, 0.29, -0.5],               # five in one bucket: general kernel
        list(np.linspace(-0.3, 0.3, 16)),
    ]
    fields, ths = [], []
    for i, t in enumerate(sets):
        shape = (int(rng.integers(20, 40)), int(rng.integers(30, 70)), int(rng.integers(33, 90)))
        f = rng.choice(np.asarray(t + [0.0, 0.55, 1.05, 0.255], dtype=dtype), size=shape)
        f = f + (rng.integers(-2, 3, size=shape) * 0.01).astype(dtype) * (rng.random(shape) < 0.5)
        f = f.astype(dtype)
        Z, Y, X = shape
        for m in (mkf.BMC_GT, mkf.BMC_GT | mkf.BMC_EQ, mkf.BMC_LT):
            got = u64(mkf.field_bpfd(to_dev(f, cuda), t, m))
            assert (got == oracle.bpfd_field(f, (X, Y, Z), t, m)).all(), (i, m)
        fields.append(to_dev(f, cuda))
        ths.append(t)
    plan = mkf.BatchPlan(fields, ths)
    want = np.concatenate([u64(mkf.field_bpfd(f, t, mkf.BMC_GT)) for f, t in zip(fields, ths)])
    assert (u64(plan.launch()) == want).all()
    plan.close()


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_three_to_six_thresholds_of_one_relation(mkf, oracle, cuda, dtype):
    """3..6 thresholds sharing one relation take the word kernel (several map words per row):
    every relation, ties and NaN, fields narrower and wider than a 32 x 32 tile."""
    rng = np.random.default_rng(23)
    for shape in [(7, 20, 45), (5, 40, 70), (9, 33, 100)]:
        f = (rng.integers(-8, 9, size=shape) * 0.25).astype(dtype)
        f.ravel()[rng.choice(f.size, f.size // 40, replace=False)] = np.nan
        Z, Y, X = shape
        for K in (3, 4, 5, 6):
            t = list(np.round(rng.uniform(-1.5, 1.5, size=K) * 4) / 4)  # on the value grid: ties
            for m in (mkf.BMC_GT, mkf.BMC_GT | mkf.BMC_EQ, mkf.BMC_LT, mkf.BMC_LT | mkf.BMC_EQ):
                got = u64(mkf.field_bpfd(to_dev(f, cuda), t, m))
                assert (got == oracle.bpfd_field(f, (X, Y, Z), t, m)).all(), (shape, K, m)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_counts_with_moments(mkf, cuda, dtype):
    """mkfFieldBPFDMoments: the counts equal mkfFieldBPFD's exactly; per threshold and map value
    the sums of f and f^2 equal FP64 sums over the elements (every element once, tiles overlap),
    within 1e-9 of the sum of magnitudes (the summation order differs)."""
    import torch

    rng = np.random.default_rng(31)
    big = to_dev(rng.standard_normal((12, 80, 150)).astype(dtype), cuda)
    cases = [rng.standard_normal(s).astype(dtype) for s in [(5, 6, 7), (3, 40, 33), (9, 64, 64), (35, 33, 97)]]
    views = [to_dev(c, cuda) for c in cases] + [big[1:11, 3:70, 5:140], big[:, :, ::2]]
    for v in views:
        f = v.cpu().numpy().astype(np.float64)
        for t, m in (([0.1], [4]), ([-0.3, 0.4], [6, 1]), ([0.2, 0.2], [2, 5]), ([0.0], [7])):
            counts, mom = mkf.field_bpfd_moments(v, t, m)
            assert (u64(counts) == u64(mkf.field_bpfd(v, t, m))).all()
            mom = mom.cpu().numpy()
            for k, (tk, mk) in enumerate(zip(t, m)):
                d = 1 - (f < tk).astype(int) + (f > tk).astype(int)
                bit = (mk >> d) & 1
                for b in (0, 1):
                    sel = f[bit == b]
                    assert abs(mom[k, b, 0] - sel.sum()) <= 1e-9 * (np.abs(f).sum() + 1)
                    assert abs(mom[k, b, 1] - (sel * sel).sum()) <= 1e-9 * ((f * f).sum() + 1)


def test_tuning_keeps_counts(mkf, cuda):
    """Slab-depth tuning changes speed only: counts before and after mkfTune, and of batch plans
    created with and without tuning, are identical."""
    import torch

    g = torch.Generator(device=cuda).manual_seed(8)
    f64 = torch.randn((150, 200, 300), dtype=torch.float64, device=cuda, generator=g)
    f32 = torch.randn((70, 90, 130), dtype=torch.float32, device=cuda, generator=g)
    cases = [(f64, np.linspace(-1.5, 1.5, 16)), (f32, [0.2]), (f32, [-0.5, 0.0, 0.5])]
    before = [u64(mkf.field_bpfd(f, t, 4)) for f, t in cases]
    for f, t in cases:
        mkf.tune(f, t, 4)
    for (f, t), b in zip(cases, before):
        assert (u64(mkf.field_bpfd(f, t, 4)) == b).all()
    # the 16-threshold FP64 field takes the TMA-staged rank-table kernel: mkfTune recorded a depth
    # and one of its variants, and every variant (CTA shape, histogram copies, queue kind) keeps
    # the counts
    depth, variant = mkf.tuned(f64, cases[0][1], 4)
    assert depth in (4, 8, 16, 32, 64, 128) and 0 <= variant < 4
    for v in range(4):
        for dep in (8, 64):
            mkf.tune(f64, cases[0][1], 4, depth=dep, variant=v)
            assert mkf.tuned(f64, cases[0][1], 4) == (dep, v)
            assert (u64(mkf.field_bpfd(f64, cases[0][1], 4)) == before[0]).all(), (v, dep)
    mkf.tune(f64, cases[0][1], 4, depth=0)
    assert mkf.tuned(f64, cases[0][1], 4) == (0, 0)
    fields = [f64, f32, f32[:40, :50, :60]]
    ths = [np.linspace(-1.5, 1.5, 16), [0.2], [0.1, 0.3]]
    plans = []
    prev = mkf.set_batch_tuning(False)
    try:
        plans.append(mkf.BatchPlan(fields, ths))
        mkf.set_batch_tuning(True)
        plans.append(mkf.BatchPlan(fields, ths))
    finally:
        mkf.set_batch_tuning(prev)
    a = u64(plans[0].launch())
    b = u64(plans[1].launch())
    assert (a == b).all()
    assert (a[:16] == before[0]).all()
    for p in plans:
        p.close()


def test_batch_fields_with_three_to_six_thresholds(mkf, oracle, cuda):
    """Batched fields with 3..6 thresholds of one relation (the rank-table batch kernel; the
    single-field calls take the word kernel up to 5 / 6 thresholds) equal the single-field counts,
    which equal the oracle's."""
    rng = np.random.default_rng(44)
    fields, ths, masks, host = [], [], [], []
    for i in range(16):
        dt = np.float32 if i % 2 else np.float64
        shape = (int(rng.integers(4, 40)), int(rng.integers(20, 70)), int(rng.integers(20, 90)))
        f = (rng.integers(-8, 9, size=shape) * 0.25).astype(dt)
        K = 3 + i % 4
        t = list(np.round(rng.uniform(-1.5, 1.5, size=K) * 4) / 4)
        m = [mkf.BMC_GT, mkf.BMC_GT | mkf.BMC_EQ, mkf.BMC_LT, mkf.BMC_LT | mkf.BMC_EQ][(i // 4) % 4]
        fields.append(to_dev(f, cuda)); ths.append(t); masks.append(m); host.append(f)
    want = []
    for f, fd, t, m in zip(host, fields, ths, masks):
        Z, Y, X = f.shape
        w = u64(mkf.field_bpfd(fd, t, m))
        assert (w == oracle.bpfd_field(f, (X, Y, Z), t, m)).all()
        want.append(w)
    plan = mkf.BatchPlan(fields, ths, masks)
    assert (u64(plan.launch()) == np.concatenate(want)).all()
    plan.close()


def test_batch_plan_with_fields_that_fill_the_gpu(mkf, cuda):
    """Fields of 2^23 voxels or more with 3+ thresholds of one relation leave the batched
    rank-table kernel for the single-field kernels inside the same plan (word kernel for a few
    thresholds, the TMA rank table on aligned rows, the global-load one on unaligned rows), with
    their constant-map thresholds; small fields stay batched. Plan launch, graph replay and the
    one-shot batch call equal the single-field counts."""
    import torch

    g = torch.Generator(device=cuda).manual_seed(91)
    big = [torch.randn((128, 256, 256), dtype=torch.float64, device=cuda, generator=g),
           torch.randn((132, 250, 258), dtype=torch.float32, device=cuda, generator=g),
           torch.randn((140, 240, 255), dtype=torch.float32, device=cuda, generator=g),  # rows off 16 B
           torch.randn((128, 256, 256), dtype=torch.float32, device=cuda, generator=g)]
    small = [torch.randn((30, 40, 50), dtype=torch.float64, device=cuda, generator=g),
             torch.randn((20, 33, 64), dtype=torch.float32, device=cuda, generator=g)]
    fields = big + small
    ths = [list(np.linspace(-1.5, 1.5, 16)), list(np.linspace(-1, 1, 8)) + [float("nan")],
           list(np.linspace(-1.2, 1.2, 12)), [-0.5, 0.0, 0.5],
           list(np.linspace(-1, 1, 9)), [-0.3, 0.1, 0.4, 0.8]]
    masks = [mkf.BMC_GT, mkf.BMC_LT | mkf.BMC_EQ, mkf.BMC_GT | mkf.BMC_EQ, mkf.BMC_LT, mkf.BMC_GT, mkf.BMC_LT]
    want = np.concatenate([u64(mkf.field_bpfd(f, t, m)) for f, t, m in zip(fields, ths, masks)])
    plan = mkf.BatchPlan(fields, ths, masks)
    assert (u64(plan.launch()) == want).all()
    assert (u64(plan.launch_graph()) == want).all()
    plan.close()
    assert (u64(mkf.batch_bpfd(fields, ths, masks)) == want).all()


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_rank_table_kernel_on_all_ones_regions(mkf, oracle, cuda, dtype):
    """Large regions above every threshold: work items of 64 (default) and 128 (tuned) planes
    whose columns are all-ones for every threshold, single-field and batched, against the oracle.
    (Their all-ones counters must hold a carry per plane: 64 planes of all-ones cells once wrapped
    a 6-slice counter.)"""
    rng = np.random.default_rng(57)
    fields, want, ths = [], [], []
    for shape in [(140, 40, 70), (200, 24, 50), (70, 33, 65)]:
        f = np.full(shape, 5.0) + rng.standard_normal(shape) * 0.01
        Z, Y, X = shape
        for _ in range(3):  # a few dips below the thresholds
            z, y, x = (int(rng.integers(0, n)) for n in shape)
            f[max(0, z - 6):z + 6, max(0, y - 6):y + 6, max(0, x - 6):x + 6] = rng.uniform(-2, 2)
        f = f.astype(dtype)
        t = list(np.linspace(-1.5, 1.5, 8))  # 8 thresholds of one relation: the rank-table kernel
        w = oracle.bpfd_field(f, (X, Y, Z), t, mkf.BMC_GT)
        fd = to_dev(f, cuda)
        assert (u64(mkf.field_bpfd(fd, t, mkf.BMC_GT)) == w).all(), shape
        mkf.tune(fd, t, mkf.BMC_GT)
        assert (u64(mkf.field_bpfd(fd, t, mkf.BMC_GT)) == w).all(), shape
        fields.append(fd); want.append(w); ths.append(t)
    plan = mkf.BatchPlan(fields, ths)
    assert (u64(plan.launch()) == np.concatenate(want)).all()
    plan.close()


def test_full_size_smooth_field_two_kernels_agree(mkf, cuda):
    """1024^3 FP64 smooth Gaussian field (sigma 4, as the benchmark's): each of the 16 rows of the
    rank-table pass equals a single-threshold pass of the word kernel (a different algorithm), at
    the default slab depth and at the tuned one. Smooth fields give long runs of all-ones cells,
    which the white-noise fields of the other full-size test never do."""
    import torch

    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if repo not in sys.path:
        sys.path.insert(0, repo)
    import bench

    f = bench.grf_torch(1024, 1024, 1024, 3, cuda)
    t = np.linspace(-2, 2, 16)
    for tuned in (False, True):
        if tuned:
            mkf.tune(f, t, mkf.BMC_GT)
        h = u64(mkf.field_bpfd(f, t, mkf.BMC_GT))
        assert (h.sum(axis=1) == 1023 ** 3).all()
        for k in range(16):
            assert (u64(mkf.field_bpfd(f, t[k:k + 1], mkf.BMC_GT))[0] == h[k]).all(), (tuned, k)
    del f
    torch.cuda.empty_cache()


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_dense_thresholds_on_a_smooth_field(mkf, oracle, cuda, dtype):
    """A smooth Gaussian field (sigma 4) with thresholds closer than its cell-to-cell variation
    (32 over [-2, 2], 16 over [-1, 1]): many cells span 4 to 7 thresholds and some 8 or more, the
    cases the rank-table kernel counts after its row loop. Whole tiles (X >= 32), single-field and
    batched, against the oracle."""
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if repo not in sys.path:
        sys.path.insert(0, repo)
    import bench

    import torch

    g = bench.grf_torch(64, 72, 160, 13, cuda)
    fd = g.to(torch.float64 if dtype == np.float64 else torch.float32).contiguous()
    f = fd.cpu().numpy()
    Z, Y, X = f.shape
    ths = [list(np.linspace(-2, 2, 32)), list(np.linspace(-1, 1, 16))]
    want = []
    for t in ths:
        w = oracle.bpfd_field(f, (X, Y, Z), t, mkf.BMC_GT)
        assert (u64(mkf.field_bpfd(fd, t, mkf.BMC_GT)) == w).all(), len(t)
        want.append(w)
    plan = mkf.BatchPlan([fd, fd], ths)
    assert (u64(plan.launch()) == np.concatenate(want)).all()
    plan.close()


def test_batch_plan_every_rank_table_variant(mkf, oracle, cuda):
    """One plan holding every variant of the batched rank-table kernel (FP32 / FP64 x relation
    > / >= x thresholds alone or sharing rank-table buckets x whole or edge-shifted tiles), which a
    launch runs as one kernel per variant over its group of chunks; against the oracle."""
    rng = np.random.default_rng(71)
    spread = [-1.2, -0.7, -0.3, 0.0, 0.2, 0.6, 0.9, 1.4]
    paired = [-0.3, -0.3001, 0.1, 0.1001, 0.5, 0.5001, 1.0, 1.0001]  # pairs share a bucket
    fields, ths, masks, want = [], [], [], []
    for dt in (np.float32, np.float64):
        for m in (mkf.BMC_GT, mkf.BMC_GT | mkf.BMC_EQ):
            for t in (spread, paired):
                for shape in ((30, 40, 45), (24, 20, 19)):  # X, Y >= 32: shifted tiles; else plain
                    f = rng.standard_normal(shape).astype(dt)
                    Z, Y, X = shape
                    want.append(oracle.bpfd_field(f, (X, Y, Z), t, m))
                    fields.append(to_dev(f, cuda)); ths.append(t); masks.append(m)
    plan = mkf.BatchPlan(fields, ths, masks)
    assert (u64(plan.launch()) == np.concatenate(want)).all()
    assert (u64(plan.launch_graph()) == np.concatenate(want)).all()
    plan.close()


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_rank_table_special_values_in_the_field(mkf, oracle, cuda, dtype):
    """NaN, +-inf and (FP64) magnitudes near the top of the range sprinkled into a field counted
    by the rank-table kernel (16 ordinary thresholds, whole tiles): those elements take the exact
    rank path, every relation of one kind, against the oracle."""
    rng = np.random.default_rng(83)
    f = rng.standard_normal((30, 48, 70))
    flat = f.ravel()
    idx = rng.choice(flat.size, 3000, replace=False)
    flat[idx[:600]] = np.nan
    flat[idx[600:1200]] = np.inf
    flat[idx[1200:1800]] = -np.inf
    if dtype == np.float64:
        flat[idx[1800:2400]] = 1e308
        flat[idx[2400:]] = -3e307
    f = f.astype(dtype)
    Z, Y, X = f.shape
    t = np.linspace(-2, 2, 16)
    for mask in (mkf.BMC_GT, mkf.BMC_GT | mkf.BMC_EQ, mkf.BMC_LT, mkf.BMC_LT | mkf.BMC_EQ):
        got = u64(mkf.field_bpfd(to_dev(f, cuda), t, mask))
        assert (got == oracle.bpfd_field(f, (X, Y, Z), t, [mask] * len(t))).all(), mask


@pytest.mark.parametrize("prof_id", [1, 2, 3])
def test_dropin_two_plane_buffer_profile(mkf, oracle, cuda, prof_id):
    """A profile with a nonzero low nibble selects the reference's small buffer layout (setBMO,
    binMapUtil.c:60-87: two rows, two planes). The drop-in maps exactly that window of the field
    (rows 0-1 of planes 0-1) and counts its one row pair of one plane pair; the reference maps the
    whole field into the small buffer there (binMapCUDA.cu:167-199), past its end."""
    rng = np.random.default_rng(90 + prof_id)
    f = rng.standard_normal((7, 9, 70)).astype(np.float32)
    fd = to_dev(f, cuda)
    pbm, org, _ = mkf.bin_map_cuda(fd, ">", 0.25, prof_id=prof_id)
    assert (org.rowPairs, org.planePairs) == (1, 1)
    got = u64(mkf.get_bpfd(pbm, org))
    sub = np.ascontiguousarray(f[:2, :2, :])
    assert (got == oracle.bpfd_field(sub, (70, 2, 2), [0.25], mkf.BMC_GT)[0]).all()


# ---------------------------------------------------------------- drop-in: maps this library did not make

def _org_of(mkf, X, Y, Z):
    import ctypes as C

    org = mkf.BMOrg()
    mkf.lib().setBMO(C.byref(org), (C.c_int * 3)(X, Y, Z), bytes([0]))
    return org


def test_dropin_counts_reference_made_maps(mkf, golden, cuda):
    """mkfCUDAGetBPFDH on the reference's own packed maps (its CPU map, binMapACC.c:43-93, as the
    golden fixtures hold them): for X % 32 != 0 their padding bits carry the next row's elements
    (binMapACC.c:86-90), which the count must ignore. Every map counts to the reference's own
    distribution. (The reference's test main counts a caller-made ENC_U1 pattern the same way,
    mkfCUDA.cu:326-331.)"""
    import torch

    n = 0
    for key in [str(v) for v in golden["names"] if not str(v).startswith("short_")]:
        Z, Y, X = golden[key + "/field"].shape
        org = _org_of(mkf, X, Y, Z)
        for k in range(golden[key + "/pbm"].shape[0]):
            words = np.ascontiguousarray(golden[key + "/pbm"][k], np.uint32)
            pbm = torch.from_numpy(words.view(np.int32).copy()).to(cuda)
            assert (mkf.get_bpfd_host(pbm, org) == golden[key + "/bpfd"][k]).all(), (key, k)
            n += 1
    assert n >= 50


@pytest.mark.parametrize("seed", range(3))
def test_dropin_counts_random_maps_with_padding_bits(mkf, oracle, cuda, seed):
    """Random packed maps, padding bits random too, several row widths: mkfCUDAGetBPFD (device,
    accumulating) and mkfCUDAGetBPFDH equal the oracle's count of the same words, which reads
    only each row's X bits; setting every padding bit changes nothing."""
    import torch

    rng = np.random.default_rng(700 + seed)
    for X in (32, 33, 63, 64, 96, 100, 257):
        Y, Z = int(rng.integers(2, 20)), int(rng.integers(2, 12))
        row, plane = layout((X, Y, Z))
        words = rng.integers(0, 1 << 32, size=plane * Z, dtype=np.uint64).astype(np.uint32)
        org = _org_of(mkf, X, Y, Z)
        want = oracle.bpfd_pbm(words, (X, Y, Z))
        assert want.sum() == (X - 1) * (Y - 1) * (Z - 1)
        pbm = torch.from_numpy(words.view(np.int32).copy()).to(cuda)
        assert (mkf.get_bpfd_host(pbm, org) == want).all(), X
        acc = mkf.get_bpfd(pbm, org)
        acc = mkf.get_bpfd(pbm, org, out=acc)
        assert (u64(acc) == 2 * want).all(), X
        padded = words | ~valid_bits_mask(X, Y, Z)
        pbm = torch.from_numpy(padded.view(np.int32).copy()).to(cuda)
        assert (mkf.get_bpfd_host(pbm, org) == want).all(), X


# ---------------------------------------------------------------- the benchmark configuration against the reference

def test_benchmark_config_equals_reference_c_path(mkf, ref_oracle, cuda):
    """The benchmark's counting pass (1024 x 1024 rows of a FP64 Gaussian random field, sigma 4,
    16 thresholds linspace(-2, 2, 16), '>') on 300 planes, against the reference's own C path
    (oracle/_ref: binMapAcc + addPlaneBPFD per z-slab on all host cores, one call per threshold)
    bit for bit, as the reference's own test compares its CPU and GPU distributions
    (mkfTest.c:64-85). Slab depths: the untuned default, the depth the benchmark's tuning keeps on
    the 1024^3 field (128 planes: two full work items and a short one along z) and the
    candidates of mkfTune, with the TMA-staged kernel's variants of CTA shape and histogram
    copies; every work item is shifted inside the field (X >= 32, Y > 8). The
    reference's interface rounds thresholds to float (binMapUtil.c:37), so both sides are given
    the float-rounded thresholds."""
    import torch

    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if repo not in sys.path:
        sys.path.insert(0, repo)
    import bench

    Z = 300
    f = bench.grf_torch(Z, 1024, 1024, 21, cuda)
    t = np.linspace(-2, 2, 16).astype(np.float32).astype(np.float64)
    host = np.ascontiguousarray(f.cpu().numpy().ravel())  # X = 1024: the reference reads no slack
    threads = max(1, len(os.sched_getaffinity(0)))
    want = np.stack([ref_oracle.bpfd_mt(host, (1024, 1024, Z), float(tv), mkf.BMC_GT, threads) for tv in t])
    assert (want.sum(axis=1) == 1023 * 1023 * (Z - 1)).all()
    del host
    for depth, variant in ((None, 0), (128, 0), (64, 0), (32, 0), (8, 0), (4, 0), (128, 1), (64, 2), (128, 3), (32, 2)):
        if depth is not None:
            mkf.tune(f, t, mkf.BMC_GT, depth=depth, variant=variant)
        got = u64(mkf.field_bpfd(f, t, mkf.BMC_GT))
        assert (got == want).all(), (depth, variant)
    mkf.tune(f, t, mkf.BMC_GT)
    assert (u64(mkf.field_bpfd(f, t, mkf.BMC_GT)) == want).all()
    mkf.tune(f, t, mkf.BMC_GT, depth=0)
    del f
    torch.cuda.empty_cache()


# ---------------------------------------------------------------- the TMA-staged rank-table kernel

def _smooth(rng, shape, dtype):
    f = rng.standard_normal(shape)
    for ax in range(3):
        f = f + np.roll(f, 1, axis=ax)
    return (f / f.std()).astype(dtype)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_tma_rank_table_kernel_against_oracle(mkf, oracle, cuda, dtype):
    """Fields whose rows start on 16-byte boundaries (X a multiple of 4 for FP32, of 2 for FP64)
    take the TMA-staged rank-table kernel for 7..16 thresholds of one relation. Every relation,
    edge items in x and y (X - 1 and Y - 1 not multiples of 31 and 8), a field of exactly one item
    row (Y = 9), a slab ending mid-item, dense thresholds (cells crossing 4 to 16 of them: the
    queued wide cells), thresholds sharing rank-table buckets (four candidates), and a view with
    aligned strides, against the oracle; no kernel wait ran out."""
    import torch

    rng = np.random.default_rng(808 if dtype == np.float64 else 809)
    a = 4 if dtype == np.float32 else 2
    shapes = [(20, 9, 32), (33, 17, 64), (12, 50, 25 * a), (9, 70, 9 * a), (130, 12, 10 * a)]
    sets = [np.linspace(-1.5, 1.5, 7), np.linspace(-2, 2, 16), np.linspace(-0.4, 0.4, 16),
            np.array([0.5, 0.5 + 1e-7, 0.5 + 2e-7, 0.5 + 3e-7, -1.0, 0.0, 1.0, 1.5])]
    masks = [mkf.BMC_GT, mkf.BMC_GT | mkf.BMC_EQ, mkf.BMC_LT, mkf.BMC_LT | mkf.BMC_EQ]
    mkf.lib().mkfKernelFaults(1)
    for i, shape in enumerate(shapes):
        f = _smooth(rng, shape, dtype)
        Z, Y, X = shape
        fd = to_dev(f, cuda)
        for j, t in enumerate(sets):
            m = masks[(i + j) % 4]
            got = u64(mkf.field_bpfd(fd, t, m))
            assert (got == oracle.bpfd_field(f, (X, Y, Z), t, m)).all(), (shape, j, m)
    # a view whose strides are multiples of 16 bytes: a sub-box of a larger field
    big = _smooth(rng, (40, 30, 16 * a), dtype)
    bd = to_dev(big, cuda)
    view = bd[3:35, 2:27, :12 * a]
    sub = np.ascontiguousarray(big[3:35, 2:27, :12 * a])
    t = np.linspace(-1.2, 1.2, 11)
    got = u64(mkf.field_bpfd(view, t, mkf.BMC_GT))
    assert (got == oracle.bpfd_field(sub, (12 * a, 25, 32), t, mkf.BMC_GT)).all()
    assert mkf.lib().mkfKernelFaults(1) == 0


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_tma_rank_table_kernel_saturated_queue_every_variant(mkf, oracle, cuda, dtype):
    """White noise under 16 thresholds spread over its range: nearly every cell crosses four or
    more thresholds, so every lane queues a wide cell in every row pair and the queues fill to
    their limit before each drain (per-lane queue: a drain after every plane; warp queue: several
    per plane). Every kernel variant, two slab depths, against the oracle; no wait ran out."""
    rng = np.random.default_rng(4242)
    shape = (40, 26, 96)
    f = rng.standard_normal(shape).astype(dtype)
    Z, Y, X = shape
    fd = to_dev(f, cuda)
    t = np.linspace(-1.6, 1.6, 16)
    want = oracle.bpfd_field(f, (X, Y, Z), t, mkf.BMC_GT)
    mkf.lib().mkfKernelFaults(1)
    for variant in range(4):
        for depth in (8, 32):
            mkf.tune(fd, t, mkf.BMC_GT, depth=depth, variant=variant)
            assert (u64(mkf.field_bpfd(fd, t, mkf.BMC_GT)) == want).all(), (variant, depth)
    mkf.tune(fd, t, mkf.BMC_GT, depth=0)
    assert mkf.lib().mkfKernelFaults(1) == 0


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_tma_rank_table_kernel_exact_path_and_depths(mkf, oracle, cuda, dtype):
    """The TMA-staged kernel's exact path: elements equal to thresholds (ties of the whole value,
    and for FP64 of the high word only), infinities, NaNs and huge magnitudes, under every relation;
    and slab depths from 4 to 255 planes (mkfTuneSet), against the oracle."""
    rng = np.random.default_rng(77)
    shape = (70, 20, 64)
    f = (rng.integers(-8, 9, size=shape) * 0.25).astype(np.float64)
    flat = f.reshape(-1)
    idx = rng.permutation(flat.size)
    flat[idx[:300]] = np.nan
    flat[idx[300:600]] = np.inf
    flat[idx[600:900]] = -np.inf
    flat[idx[900:1000]] = 1e300 if dtype == np.float64 else 3e38
    flat[idx[1000:1400]] = 0.5 + 1e-12  # same FP64 high word as 0.5
    f = f.astype(dtype)
    Z, Y, X = shape
    fd = to_dev(f, cuda)
    t = np.arange(-1.75, 2.0, 0.25)  # 15 thresholds on the values' grid: many exact ties
    for m in (mkf.BMC_GT, mkf.BMC_GT | mkf.BMC_EQ, mkf.BMC_LT, mkf.BMC_LT | mkf.BMC_EQ):
        want = oracle.bpfd_field(f, (X, Y, Z), t, m)
        assert (u64(mkf.field_bpfd(fd, t, m)) == want).all(), m
    want = oracle.bpfd_field(f, (X, Y, Z), t, mkf.BMC_GT)
    for depth in (4, 8, 64, 128, 255):
        mkf.tune(fd, t, mkf.BMC_GT, depth=depth)
        assert (u64(mkf.field_bpfd(fd, t, mkf.BMC_GT)) == want).all(), depth
    mkf.tune(fd, t, mkf.BMC_GT, depth=0)
    assert mkf.lib().mkfKernelFaults(1) == 0

