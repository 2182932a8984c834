"""The library's host-side launch logic on the CPU (twins_b200/csrc/tb_host.h, built here with g++
through the shim tests/host_logic.cpp): the launch-shape tuner's start rule, hysteresis and
strikes, the running-unit lists of a batch, the grid rule, and the server's first-fit ranges
against a plain model of each."""
import ctypes as C
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT

SHIM = ROOT / "tests" / "host_logic.cpp"
CSRC = ROOT / "twins_b200" / "csrc"


@pytest.fixture(scope="module")
def hl(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ is not here")
    so = tmp_path_factory.mktemp("hl") / "libhl.so"
    subprocess.run(["g++", "-std=c++17", "-O1", "-shared", "-fPIC", f"-I{CSRC}", "-o", str(so), str(SHIM)], check=True)
    lib = C.CDLL(str(so))
    vp, ll, ull = C.c_void_p, C.c_longlong, C.c_ulonglong
    sig = {
        "hl_stage": (C.c_int, [C.c_int]),
        "hl_n_cand": (C.c_int, []),
        "hl_cand": (None, [C.c_int, C.POINTER(C.c_int)]),
        "hl_grid_of": (C.c_int, [ll, C.c_int, C.c_int, C.c_int, C.c_int]),
        "hl_running_units": (C.c_int, [C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.c_int]),
        "hl_tuner": (vp, [C.c_int, C.c_int, C.c_int, C.c_int, ll, C.c_int, ll, C.c_uint]),
        "hl_tuner_free": (None, [vp]),
        "hl_tuner_n": (C.c_int, [vp]),
        "hl_tuner_shape": (None, [vp, C.c_int, C.POINTER(C.c_int)]),
        "hl_tuner_best": (C.c_int, [vp]),
        "hl_tuner_explore": (C.c_int, [vp]),
        "hl_tuner_probes": (C.c_int, [vp, C.c_int]),
        "hl_tuner_period": (C.c_int, [vp]),
        "hl_tuner_backoff": (None, [vp, C.c_int]),
        "hl_tuner_load_changed": (None, [vp]),
        "hl_tuner_tick": (None, [vp]),
        "hl_tuner_add_slots": (None, [vp, C.c_int, ll]),
        "hl_tuner_most": (C.c_int, [vp]),
        "hl_tuner_decide": (None, [vp, C.POINTER(C.c_double)]),
        "hl_ranges": (vp, [ull]),
        "hl_ranges_free": (None, [vp]),
        "hl_take": (ll, [vp, ull]),
        "hl_give": (None, [vp, ull, ull]),
        "hl_used": (ull, [vp]),
        "hl_free_ranges": (C.c_int, [vp, C.POINTER(ull), C.c_int]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    return lib


SMALL, MID, TWO, MAX = 96, 192, 288, 384


def test_staging_sizes_and_candidates(hl):
    assert [hl.hl_stage(i) for i in range(4)] == [SMALL, MID, TWO, MAX]
    cands = []
    for k in range(hl.hl_n_cand()):
        v = (C.c_int * 3)()
        hl.hl_cand(k, v)
        cands.append(tuple(v))
    assert len(set(cands)) == len(cands)
    for lanes, stage, pl in cands:
        assert lanes in (1, 4, 32) and 1 <= stage <= MAX
        assert not pl or lanes == 1  # the port-local egress runs with one host per warp only


def test_grid_rule(hl):
    g = hl.hl_grid_of
    assert g(0, 4, 2, 148, 0) == 1  # an empty batch still launches one block
    assert g(10, 4, 2, 148, 0) == 3
    assert g(10_000, 4, 2, 148, 0) == 296  # capped at what is co-resident
    assert g(10, 4, 0, 148, 0) == 0  # the shape does not fit
    assert g(10, 4, 2, 148, 50) == 50 and g(10, 4, 2, 148, 1000) == 296  # the caller's grid, capped


def tuner(hl, entities, kmax=8, resident=1184, mask=0x1FF, autotune=True, fixed=(1, MID, 0)):
    t = hl.hl_tuner(int(autotune), fixed[0], fixed[1], fixed[2], entities, kmax, resident, mask)
    shapes = []
    for k in range(hl.hl_tuner_n(t)):
        v = (C.c_int * 4)()
        hl.hl_tuner_shape(t, k, v)
        shapes.append(tuple(v))
    return t, shapes


def test_tuner_start_rule(hl):
    # few entities for the resident warps: one host per warp, two blocks per SM
    t, shapes = tuner(hl, 208)
    assert len(shapes) == 9 and shapes[hl.hl_tuner_best(t)][:3] == (1, TWO, 0)
    hl.hl_tuner_free(t)
    # big switches: the port-local egress with the largest staging
    t, shapes = tuner(hl, 208, kmax=16)
    assert shapes[hl.hl_tuner_best(t)][:3] == (1, MAX, 1)
    hl.hl_tuner_free(t)
    # many entities: 32 hosts per warp with the smallest staging (the rule is on entities <= 2x resident)
    t, shapes = tuner(hl, 2 * 1184 + 1, kmax=32)
    assert shapes[hl.hl_tuner_best(t)][:3] == (32, SMALL, 0)
    hl.hl_tuner_free(t)
    t, shapes = tuner(hl, 2 * 1184)
    assert shapes[hl.hl_tuner_best(t)][:3] == (1, TWO, 0)
    hl.hl_tuner_free(t)


def test_tuner_candidates_that_fit_and_fixed_shape(hl):
    # only the candidates the device fits are kept; a start shape that does not fit falls back to the first
    t, shapes = tuner(hl, 208, mask=0b0000_1110)
    assert [s[:3] for s in shapes] == [(1, MID, 0), (4, MID, 0), (32, MID, 0)] and hl.hl_tuner_best(t) == 0
    hl.hl_tuner_free(t)
    # no autotuning, or nothing fits: the caller's shape alone, never probed
    for kw in ({"autotune": False}, {"mask": 0}):
        t, shapes = tuner(hl, 208, fixed=(4, SMALL, 0), **kw)
        assert [s[:3] for s in shapes] == [(4, SMALL, 0)]
        for _ in range(100):
            hl.hl_tuner_tick(t)
        assert not hl.hl_tuner_explore(t)
        hl.hl_tuner_free(t)


def decide(hl, t, per_slot):
    arr = (C.c_double * len(per_slot))(*per_slot)
    hl.hl_tuner_decide(t, arr)


def test_tuner_hysteresis_strikes_and_expiry(hl):
    t, shapes = tuner(hl, 208)
    n = len(shapes)
    b0 = hl.hl_tuner_best(t)
    period = hl.hl_tuner_period(t)
    for i in range(period):
        assert not hl.hl_tuner_explore(t)
        hl.hl_tuner_tick(t)
    assert hl.hl_tuner_explore(t)
    # a shape 4% faster does not take over; every shape more than 30% slower takes a strike, and
    # one more than 60% slower two (it is not probed again)
    ps = [1.0 if k == b0 else 1.4 for k in range(n)]
    other = (b0 + 1) % n
    far = (b0 + 2) % n
    ps[other], ps[far] = 0.96, 1.7
    decide(hl, t, ps)
    assert hl.hl_tuner_best(t) == b0 and not hl.hl_tuner_explore(t)
    assert not hl.hl_tuner_probes(t, far)
    assert all(hl.hl_tuner_probes(t, k) for k in range(n) if k != far)
    # second round: 6% faster takes over, and the slow ones take their second strike
    ps[other] = 0.94
    decide(hl, t, ps)
    assert hl.hl_tuner_best(t) == other
    slow = [k for k in range(n) if ps[k] >= 1.4]
    assert slow and all(not hl.hl_tuner_probes(t, k) for k in slow)
    assert hl.hl_tuner_probes(t, b0) and hl.hl_tuner_probes(t, other)
    # rounds 3 and 4 without probes of the struck shapes; the fourth round clears every strike
    skip = [ps[k] if hl.hl_tuner_probes(t, k) else -1 for k in range(n)]
    decide(hl, t, skip)
    assert all(not hl.hl_tuner_probes(t, k) for k in slow)
    decide(hl, t, skip)
    assert all(hl.hl_tuner_probes(t, k) for k in range(n))
    hl.hl_tuner_free(t)


def test_tuner_backoff(hl):
    t, shapes = tuner(hl, 208)
    n = len(shapes)
    p0 = hl.hl_tuner_period(t)
    # without backoff the period stays
    decide(hl, t, [1.0] * n)
    assert hl.hl_tuner_period(t) == p0
    hl.hl_tuner_backoff(t, 4 * p0)
    b0 = hl.hl_tuner_best(t)
    keep = [1.0 if k == b0 else 1.2 for k in range(n)]
    periods = []
    for _ in range(4):
        decide(hl, t, keep)
        periods.append(hl.hl_tuner_period(t))
    assert periods == [2 * p0, 4 * p0, 4 * p0, 4 * p0] and hl.hl_tuner_best(t) == b0
    # a change of the load restores the first period and clears the strikes; a new shape restores the period
    far = [1.0 if k == b0 else 2.0 for k in range(n)]
    decide(hl, t, far)
    assert all(not hl.hl_tuner_probes(t, k) for k in range(n) if k != b0)
    hl.hl_tuner_load_changed(t)
    assert hl.hl_tuner_period(t) == p0
    assert all(hl.hl_tuner_probes(t, k) for k in range(n))
    decide(hl, t, keep)
    assert hl.hl_tuner_period(t) == 2 * p0
    new = list(keep)
    new[(b0 + 1) % n] = 0.5
    decide(hl, t, new)
    assert hl.hl_tuner_best(t) == (b0 + 1) % n and hl.hl_tuner_period(t) == p0
    hl.hl_tuner_free(t)


def test_tuner_unprobed_best_and_most(hl):
    t, shapes = tuner(hl, 208)
    n = len(shapes)
    # the running shape's probe ran too few slots (<= 0): the fastest probed shape takes over
    ps = [-1.0] * n
    ps[2], ps[5] = 3.0, 2.0
    decide(hl, t, ps)
    assert hl.hl_tuner_best(t) == 5
    for k, s in [(0, 100), (3, 500), (5, 499)]:
        hl.hl_tuner_add_slots(t, k, s)
    assert hl.hl_tuner_most(t) == 3
    hl.hl_tuner_free(t)


def units_model(alive, worlds, lanes, H):
    hu = -(-H // lanes)
    host = sorted({h // lanes for w, (h0, nh, _, _) in enumerate(worlds) if alive[w] for h in range(h0, h0 + nh)})
    sw = [hu + s0 + x for w, (_, _, s0, ns) in enumerate(worlds) if alive[w] for x in range(ns)]
    return host + sw


@pytest.mark.parametrize("seed", range(6))
def test_running_units(hl, seed):
    rng = np.random.default_rng(seed)
    W = int(rng.integers(1, 40))
    worlds, h, s = [], 0, 0
    for _ in range(W):
        nh, ns = int(rng.integers(0, 70)), int(rng.integers(0, 12))
        worlds.append((h, nh, s, ns))
        h, s = h + nh, s + ns
    for lanes in (1, 4, 32):
        alive = rng.integers(0, 2, W)
        flat = (C.c_int * (4 * W))(*[x for w in worlds for x in w])
        out = (C.c_int * (h + s + 1))()
        n = hl.hl_running_units((C.c_int * W)(*alive.tolist()), flat, W, lanes, h, out, len(out))
        assert list(out[:n]) == units_model(alive, worlds, lanes, h)


@pytest.mark.parametrize("seed", range(4))
def test_ranges_first_fit(hl, seed):
    rng = np.random.default_rng(100 + seed)
    cap = 300
    r = hl.hl_ranges(cap)
    taken = np.zeros(cap, bool)
    held = []
    for _ in range(3000):
        if held and rng.random() < 0.45:
            at, n = held.pop(int(rng.integers(len(held))))
            hl.hl_give(r, at, n)
            taken[at:at + n] = False
        else:
            n = int(rng.integers(0, 40))
            at = hl.hl_take(r, n)
            # the model: the lowest start of n free entries
            want = -1 if n else 0
            if n:
                run = 0
                for i in range(cap):
                    run = run + 1 if not taken[i] else 0
                    if run == n:
                        want = i - n + 1
                        break
            assert at == want
            if at >= 0 and n:
                taken[at:at + n] = True
                held.append((at, n))
        assert hl.hl_used(r) == taken.sum()
        buf = (C.c_ulonglong * (2 * cap))()
        m = hl.hl_free_ranges(r, buf, cap)
        ranges = [(buf[2 * i], buf[2 * i + 1]) for i in range(m)]
        # the free ranges are exactly the free entries, each maximal (none adjacent to the next)
        free = np.zeros(cap, bool)
        for a, ln in ranges:
            assert ln > 0 and not free[a:a + ln].any()
            free[a:a + ln] = True
        assert (free == ~taken).all()
        assert all(a1 + l1 < a2 for (a1, l1), (a2, _) in zip(ranges, ranges[1:]))
    for at, n in held:
        hl.hl_give(r, at, n)
    buf = (C.c_ulonglong * 2)()
    assert hl.hl_free_ranges(r, buf, 1) == 1 and (buf[0], buf[1]) == (0, cap) and hl.hl_used(r) == 0
    hl.hl_ranges_free(r)
