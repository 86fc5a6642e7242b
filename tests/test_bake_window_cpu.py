"""The windowed form of the bone bake's sequential nearest-triangle rule, on the CPU.

The reference keeps per voxel, in triangle order, a running minimum R of the
accepted squared distances and the last accepted triangle; a triangle is
accepted when d + eps(R) < R, or when |d - R| <= eps(R) with a larger
|projection| (eps(R) = 1e-7 max(1, R); bake_sdf.wgsl:131-183).  k_bone_bake
computes m = min d first and then runs the rule only over the window
{d <= m + W}, from the window's first "hard record" (a member below the window
top, and below every earlier member, by more than 1e-6 max(1, qmin)); a window
without one is retried four times wider, three times, before the full scan.

These tests restate both forms in float32 and check that they end in the same
state on sequences built to stress the argument: dense near-ties, slow
descents in steps inside the tolerance, exact duplicates, NaN and huge values.
"""
import numpy as np
import pytest

F = np.float32


def _accept(R, A, d, a):
    eps = F(1e-7) * max(F(1), R)
    closer = F(d + eps) < R
    tie = abs(F(d - R)) <= eps and a > A
    return closer or tie


def full_rule(ds, aps):
    R, A, last = F(1e10), F(-1), -1
    for t, (d, a) in enumerate(zip(ds, aps)):
        if _accept(R, A, d, a):
            if d < R:
                R = d
            A, last = a, t
    return R, A, last


def windowed_rule(ds, aps):
    finite = [d for d in ds if d == d]
    m = min(finite) if finite else F(1e30)
    W = F(4e-6) * max(F(1), m)
    for _ in range(4):
        T = F(m + W)
        R, A, last, started, qmin = F(1e10), F(-1), -1, False, T
        for t, (d, a) in enumerate(zip(ds, aps)):
            if not (d <= T):
                continue
            if started:
                pass
            elif F(d + F(1e-6) * max(F(1), qmin)) < qmin:
                started = True
            else:
                qmin = min(qmin, d)
                continue
            if _accept(R, A, d, a):
                if d < R:
                    R = d
                A, last = a, t
        if started:
            return R, A, last
        W = F(W * F(4))
    return full_rule(ds, aps)


def _check(ds, aps):
    ds = np.asarray(ds, F)
    aps = np.asarray(aps, F)
    assert windowed_rule(list(ds), list(aps)) == full_rule(list(ds), list(aps))


@pytest.mark.parametrize("seed", range(40))
def test_dense_near_ties(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 400))
    base = F(10.0 ** rng.uniform(-8, -1))
    ds = base + rng.integers(0, 40, n).astype(F) * F(rng.choice([2.5e-8, 5e-8, 1e-7, 3e-7]))
    ds = np.where(rng.random(n) < 0.3, ds + F(rng.uniform(0, 1e-3)), ds)
    _check(ds, rng.random(n).astype(F))


@pytest.mark.parametrize("seed", range(20))
def test_slow_descents_inside_the_tolerance(seed):
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(50, 600))
    step = F(rng.choice([2e-8, 6e-8, 9e-8, 2e-7, 9e-7]))
    start = F(10.0 ** rng.uniform(-6, -2))
    ds = (start - np.arange(n, dtype=F) * step).astype(F)
    ds = np.maximum(ds, F(0))
    if seed % 2:
        ds = ds[::-1].copy()
    _check(ds, rng.random(n).astype(F))


@pytest.mark.parametrize("seed", range(20))
def test_duplicates_nan_and_huge(seed):
    rng = np.random.default_rng(200 + seed)
    n = int(rng.integers(1, 200))
    ds = rng.choice(np.asarray([0.0, 1e-8, 1e-7, 2e-7, 1e-4, 1e-4 + 1e-7, 0.5, 2.0, 1e12, np.nan], F), n)
    aps = rng.choice(np.asarray([0.0, 0.1, 0.1, 0.5, 1.0], F), n)
    _check(ds, aps)


def test_window_can_start_late_and_widen():
    # the first window member sits at its top: no hard record until a wider window
    ds = [F(1.0e-4 + 3.9e-6), F(1.0e-4 + 3.5e-6), F(1.0e-4 + 3.1e-6), F(1.0e-4 + 2.7e-6), F(1.0e-4)]
    aps = [F(0.5), F(0.4), F(0.9), F(0.1), F(0.2)]
    _check(ds, aps)
