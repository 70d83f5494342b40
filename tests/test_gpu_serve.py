"""The request loop (mkfServer*): every result must be the same when its request runs alone and
when it is packed with others into shared launches, and equal to the single-field call (itself
checked against the oracle); admission must respect the device-memory budget."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _items(mkf, cuda, seed, n):
    import torch

    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        if i % 11 == 5:
            shape = (int(rng.integers(100, 160)), int(rng.integers(100, 200)), int(rng.integers(90, 260)))
        else:
            shape = tuple(int(v) for v in rng.integers(3, 70, size=3))
        dt = np.float32 if rng.random() < 0.7 else np.float64
        f = (rng.integers(-6, 7, size=shape) * 0.25 + rng.standard_normal(shape) * 0.01 * (i % 2)).astype(dt)
        K = int(rng.integers(1, 9))
        t = np.round(rng.uniform(-1.2, 1.2, size=K), 2)
        kind = i % 5
        if kind == 0:
            m = mkf.BMC_GT
        elif kind == 1:
            m = mkf.BMC_LT | mkf.BMC_EQ
        elif kind == 2:
            m = [int(v) for v in rng.integers(0, 8, size=K)]  # mixed relations and constant maps
        elif kind == 3:
            m = mkf.BMC_GT | mkf.BMC_EQ
        else:
            m = mkf.BMC_LT
        host = i % 3 == 1
        fd = torch.from_numpy(f).to(cuda)
        src = torch.from_numpy(f).pin_memory() if host else fd
        want = mkf.field_bpfd(fd, t, m).cpu().numpy().view(np.uint64).copy()
        out.append({"f": f, "src": src, "t": t, "m": m, "want": want, "host_out": i % 4 == 0})
    return out


def _run(srv, it):
    tk = srv.submit(it["src"], it["t"], it["m"], host_out=it["host_out"])
    return tk


def _result(srv, it, tk):
    res, lat = srv.wait(tk, timeout=120)
    if it["host_out"]:
        return res, lat
    got = srv.counts(tk)
    srv.release(tk)
    return got, lat


def test_server_results_alone_and_in_mix(mkf, oracle, cuda):
    items = _items(mkf, cuda, 7, 40)
    for it in items[:6]:
        Z, Y, X = it["f"].shape
        if it["f"].size < 40000:
            assert (it["want"] == oracle.bpfd_field(it["f"], (X, Y, Z), it["t"], it["m"])).all()
    srv = mkf.Server(hbm_budget=1 << 30)
    try:
        alone = []
        for it in items:
            got, lat = _result(srv, it, _run(srv, it))
            assert (got == it["want"]).all()
            assert lat > 0
            alone.append(got)
        st = srv.stats(reset=True)
        assert st["completed"] == len(items) and st["failed"] == 0

        # the same requests from three threads at once, then waited for in reverse order
        tickets = [None] * len(items)

        def producer(k):
            for i in range(k, len(items), 3):
                tickets[i] = _run(srv, items[i])

        th = [threading.Thread(target=producer, args=(k,)) for k in range(3)]
        for x in th:
            x.start()
        for x in th:
            x.join()
        for i in reversed(range(len(items))):
            got, _ = _result(srv, items[i], tickets[i])
            assert (got == alone[i]).all(), i
        st = srv.stats()
        assert st["completed"] == len(items) and st["failed"] == 0
        assert st["launches"] < len(items) and st["maxFieldsInLaunch"] > 1  # requests shared launches
        assert 0 < st["p50"] <= st["p99"] <= st["max"]
        assert st["deviceBytesInUse"] == 0
    finally:
        srv.close()


def test_server_budget_admission(mkf, cuda):
    import torch

    rng = np.random.default_rng(3)
    budget = 8 << 20
    srv = mkf.Server(hbm_budget=budget, max_fields_per_launch=4)
    try:
        # ten 3 MB pinned host fields through an 8 MB budget: at most two are staged at a time
        fields = [torch.from_numpy(rng.standard_normal((30, 100, 250)).astype(np.float32)).pin_memory() for _ in range(10)]
        want = [mkf.field_bpfd(f.to(cuda), [0.0, 0.5], mkf.BMC_GT).cpu().numpy().view(np.uint64) for f in fields]
        tks = [srv.submit(f, [0.0, 0.5], mkf.BMC_GT, host_out=True) for f in fields]
        for tk, w in zip(tks, want):
            got, _ = srv.wait(tk, timeout=120)
            assert (got == w).all()
        # a request that can never fit is refused, and the server keeps serving
        big = torch.zeros((40, 256, 256), dtype=torch.float32).pin_memory()  # 10.5 MB
        tk = srv.submit(big, [0.0], mkf.BMC_GT, host_out=True)
        with pytest.raises(mkf.MKFError, match="budget"):
            srv.wait(tk, timeout=60)
        srv.release(tk)
        tk = srv.submit(fields[0], [0.0, 0.5], mkf.BMC_GT, host_out=True)
        got, _ = srv.wait(tk, timeout=60)
        assert (got == want[0]).all()
        st = srv.stats()
        assert st["failed"] == 1 and st["deviceBytesInUse"] == 0
    finally:
        srv.close()


def test_server_shutdown_with_unreleased_counts(mkf, cuda):
    """Counts the client never releases keep their budget; closing the server must not wait for
    requests that can no longer fit."""
    import threading

    import torch

    f = torch.randn((20, 30, 40), device=cuda)
    t = list(np.linspace(-1, 1, 32))  # 32 x 256 x 8 B = 64 KiB of counts per request
    srv = mkf.Server(hbm_budget=1 << 20)
    tks = [srv.submit(f, t, mkf.BMC_GT) for _ in range(20)]
    for tk in tks[:16]:  # 16 x 64 KiB fill the 1 MiB budget
        srv.wait(tk, timeout=60)
    with pytest.raises(mkf.MKFError, match="TIMEOUT"):
        srv.wait(tks[16], timeout=0.5)
    done = threading.Event()
    th = threading.Thread(target=lambda: (srv.close(), done.set()))
    th.start()
    th.join(timeout=60)
    assert done.is_set(), "server shutdown waited for requests that cannot fit"
