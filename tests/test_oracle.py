"""The oracle pinned against the reference: golden vectors, known answers, and cross-checks.

CPU only. The golden vectors were produced by the reference MKF C path itself
(tests/golden/make_golden.py); the reference library is also compared directly where it is built.
"""
import itertools

import numpy as np
import pytest

from oracle import bpfd_numpy, layout


def valid_bits_mask(X, Y, Z):
    row, _ = layout((X, Y, Z))
    m = np.zeros(row, np.uint32)
    for w in range(row):
        nb = min(32, X - 32 * w)
        m[w] = np.uint32((1 << nb) - 1) if nb < 32 else np.uint32(0xFFFFFFFF)
    return np.tile(m, Y * Z)


def golden_cases(golden):
    return [str(n) for n in golden["names"] if not str(n).startswith("short_")]


def orbit_partition():
    """Orbits of the 256 cell patterns under the 48 symmetries of the cube (axis permutations x
    reflections), computed independently of any table."""
    perms = []
    for axes in itertools.permutations(range(3)):
        for refl in range(8):
            p = []
            for i in range(8):
                c = [(i >> a) & 1 for a in range(3)]
                d = [c[axes[a]] ^ ((refl >> a) & 1) for a in range(3)]
                p.append(d[0] | (d[1] << 1) | (d[2] << 2))
            perms.append(p)
    orbit = list(range(256))
    for pat in range(256):
        imgs = []
        for p in perms:
            q = 0
            for i in range(8):
                if (pat >> i) & 1:
                    q |= 1 << p[i]
            imgs.append(q)
        orbit[pat] = min(imgs)
    return orbit


def test_group_map_is_reference_table(oracle, golden):
    assert (oracle.group_map() == golden["c8s_map"]).all()


def test_group_map_is_cube_symmetry_orbits(oracle):
    g = oracle.group_map()
    orb = orbit_partition()
    assert len(set(orb)) == 22
    for a in range(256):
        for b in range(a + 1, 256):
            assert (g[a] == g[b]) == (orb[a] == orb[b])


@pytest.mark.parametrize("idx", range(8))
def test_oracle_matches_golden_counts(oracle, golden, idx):
    names = golden_cases(golden)
    if idx >= len(names):
        pytest.skip("no case")
    key = names[idx]
    f = golden[key + "/field"]
    Z, Y, X = f.shape
    t, m = golden[key + "/t"], golden[key + "/m"]
    want = golden[key + "/bpfd"]
    got = oracle.bpfd_field(f, (X, Y, Z), t, m)
    assert (got == want).all(), key
    # the packed map agrees on every element bit (padding bits excluded)
    vm = valid_bits_mask(X, Y, Z)
    for k in range(len(t)):
        pb = oracle.pack(f, (X, Y, Z), t[k], m[k])
        assert ((pb & vm) == (golden[key + "/pbm"][k] & vm)).all()
        assert (oracle.bpfd_pbm(pb, (X, Y, Z)) == want[k]).all()
    # single-precision measures of the reference
    for k in range(len(t)):
        rv, mm, sym = oracle.select_measures(want[k], 3.0 / (X + Y + Z))
        assert rv == 2 and sym == b"Kv       Vv\x00"
        assert mm.tobytes() == golden[key + "/sel_m"][k].tobytes()


def test_remaining_golden_cases(oracle, golden):
    for key in golden_cases(golden)[8:]:
        f = golden[key + "/field"]
        Z, Y, X = f.shape
        got = oracle.bpfd_field(f, (X, Y, Z), golden[key + "/t"], golden[key + "/m"])
        assert (got == golden[key + "/bpfd"]).all(), key


def test_short_rows_differ_from_reference_as_documented(oracle, golden):
    """Rows shorter than 32 elements: the reference counts 2X-1 cells per row (mkfACC.c:137-150);
    this build counts X-1, like every longer row."""
    for key in [str(n) for n in golden["names"] if str(n).startswith("short_")]:
        f = golden[key + "/field"]
        Z, Y, X = f.shape
        ref = golden[key + "/ref_short_bpfd"]
        ours = oracle.bpfd_field(f, (X, Y, Z), 0.0, 4)[0]
        assert int(ours.sum()) == max(X - 1, 0) * (Y - 1) * (Z - 1)
        if X > 1:
            assert int(ref.sum()) == (2 * X - 1) * (Y - 1) * (Z - 1)
        assert (ours == bpfd_numpy(f, 0.0, 4)).all()


@pytest.mark.parametrize("seed", range(6))
def test_oracle_vs_numpy_random(oracle, seed):
    rng = np.random.default_rng(seed)
    for _ in range(6):
        X, Y, Z = (int(rng.integers(1, 70)), int(rng.integers(1, 9)), int(rng.integers(1, 7)))
        f = rng.integers(-3, 4, size=(Z, Y, X)).astype(np.float64) * 0.5
        t = float(rng.choice([-0.5, 0.0, 0.5, 1.0]))
        m = int(rng.integers(0, 8))
        assert (oracle.bpfd_field(f, (X, Y, Z), t, m)[0] == bpfd_numpy(f, t, m)).all()
        pb = oracle.pack(f, (X, Y, Z), t, m)
        assert (oracle.bpfd_pbm(pb, (X, Y, Z)) == bpfd_numpy(f, t, m)).all()


@pytest.mark.parametrize("seed", range(4))
def test_oracle_vs_reference_library(oracle, ref_oracle, seed):
    rng = np.random.default_rng(100 + seed)
    for _ in range(8):
        X, Y, Z = (int(rng.integers(32, 130)), int(rng.integers(2, 10)), int(rng.integers(2, 8)))
        f = rng.standard_normal((Z, Y, X))
        f[rng.random(f.shape) < 0.05] = 0.25
        t = float(np.float32(0.25))
        m = int(rng.integers(0, 8))
        want = ref_oracle.bpfd_simple(f, (X, Y, Z), t, m)
        assert (oracle.bpfd_field(f, (X, Y, Z), t, m)[0] == want).all()
        assert (ref_oracle.bpfd_mt(ref_oracle.padded(f), (X, Y, Z), t, m, 3) == want).all()


def test_cells_sum_and_uniform_fields(oracle):
    for X, Y, Z in [(5, 4, 3), (33, 2, 2), (64, 3, 5), (1, 9, 9), (40, 1, 3)]:
        cells = max(X - 1, 0) * max(Y - 1, 0) * max(Z - 1, 0)
        ones = np.ones((Z, Y, X))
        h1 = oracle.bpfd_field(ones, (X, Y, Z), 0.5, 4)[0]
        h0 = oracle.bpfd_field(ones, (X, Y, Z), 2.0, 4)[0]
        assert int(h1.sum()) == cells and int(h1[255]) == cells
        assert int(h0.sum()) == cells and int(h0[0]) == cells


def _ball(n, centres, r, hollow=None):
    z, y, x = np.meshgrid(*(np.arange(n, dtype=np.float64),) * 3, indexing="ij")
    f = np.full((n, n, n), -1e9)
    for c in centres:
        d = np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2)
        g = r - d
        if hollow:
            g = np.minimum(g, d - hollow)
        f = np.maximum(f, g)
    return f


def test_euler_characteristic_known_answers(oracle):
    """chi = 1 for a ball, 2 for two disjoint balls, 2 for a ball with a cavity, 0 for a torus."""
    n = 40
    cases = [
        (_ball(n, [(19.5, 19.5, 19.5)], 12.0), 1),
        (_ball(n, [(10.5, 10.5, 19.5), (29.5, 29.5, 19.5)], 7.0), 2),
        (_ball(n, [(19.5, 19.5, 19.5)], 14.0, hollow=6.0), 2),
    ]
    z, y, x = np.meshgrid(*(np.arange(n, dtype=np.float64),) * 3, indexing="ij")
    rho = np.sqrt((x - 19.5) ** 2 + (y - 19.5) ** 2)
    cases.append((4.0 - np.sqrt((rho - 11.0) ** 2 + (z - 19.5) ** 2), 0))
    for f, chi in cases:
        h = oracle.bpfd_field(f, (n, n, n), 0.0, 4)[0]
        r = oracle.measures(h)
        assert r[3] == chi
        assert r[0] == float(sum(int(h[c]) for c in range(1, 256, 2)))


def test_measures_formula(oracle):
    rng = np.random.default_rng(7)
    h = rng.integers(0, 10**9, size=256).astype(np.uint64)
    g = np.zeros(22, np.uint64)
    gm = oracle.group_map()
    for c in range(256):
        g[gm[c]] += h[c]
    wk, ws, wm = oracle.weights()
    r = oracle.measures(h)
    s = float(g[0]) * ws[0]
    mc = float(g[0]) * wm[0]
    for i in range(1, 22):
        s += float(g[i]) * ws[i]
        mc += float(g[i]) * wm[i]
    assert r[1] == s and r[2] == mc
    assert r[3] == int(sum(int(wk[i]) * int(g[i]) for i in range(22))) / 24.0
