"""GPU primitives against NumPy and the oracle (needs a GPU).

The radix-sort and kNN cases are the reference's own (tests/test_msplat.py:429-465):
stable sort vs np.argsort(kind="stable"), exact 3-NN vs float64 brute force with
rtol 1e-4 on uniform, "street" (thin road plane, facade, far outliers) and duplicate
clouds. Densification, opacity reset and Gaussian initialisation are compared with
the CPU oracle on seeded inputs.
"""
import numpy as np
import pytest
import torch

from msplat_street_b200 import _core, scenes
from msplat_street_b200.backend import Context
from oracle_lib import Oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,bits,hi", [
    (1, 32, 10), (5, 32, 4), (1023, 32, 2 ** 30), (1024, 32, 2 ** 30), (1025, 32, 7),
    (70_000, 32, 2 ** 30), (5_000, 64, 2 ** 63), (2_049, 64, 3),
    (1_000_003, 43, 2 ** 43), (300_000, 30, 2 ** 40), (2_500_000, 64, 2 ** 62), (5_000_001, 40, 2 ** 40),
])
def test_gpu_radix_sort_matches_numpy(n, bits, hi):
    rng = np.random.default_rng(n + bits)
    keys = rng.integers(0, hi, n, dtype=np.uint64)
    sorted_keys, order = _core._gpu_radix_sort(keys, bits)
    mask = np.uint64((1 << bits) - 1) if bits < 64 else np.uint64(2 ** 64 - 1)
    ref = np.argsort(keys & mask, kind="stable")
    np.testing.assert_array_equal(sorted_keys, keys[ref])
    np.testing.assert_array_equal(order, ref)  # stable


def test_gpu_radix_sort_empty():
    k, v = _core._gpu_radix_sort(np.zeros(0, np.uint64), 32)
    assert k.size == 0 and v.size == 0


def _knn3_bruteforce(pts):
    d2 = ((pts[:, None, :].astype(np.float64) - pts[None, :, :]) ** 2).sum(-1)
    np.fill_diagonal(d2, np.inf)
    return np.sqrt(np.sort(d2, axis=1)[:, :3]).mean(axis=1)


def _clouds():
    rng = np.random.default_rng(7)
    road = np.c_[rng.uniform(-20, 20, 2000), rng.normal(0, 0.02, 2000), rng.uniform(0, 80, 2000)]
    facade = np.c_[8 + rng.normal(0, 0.05, 800), rng.uniform(0, 10, 800), rng.uniform(0, 80, 800)]
    return {
        "uniform": rng.uniform(-1, 1, (3000, 3)),
        "street": np.vstack([road, facade, rng.normal(0, 300, (200, 3))]),
        "duplicates": np.vstack([rng.uniform(-1, 1, (500, 3)), np.repeat(rng.uniform(-1, 1, (8, 3)), 4, axis=0)]),
    }


@pytest.mark.parametrize("kind", ["uniform", "street", "duplicates"])
def test_gpu_knn_matches_bruteforce(kind):
    pts = _clouds()[kind].astype(np.float32)
    got = _core._gpu_knn3_mean_dist(pts)
    np.testing.assert_allclose(got, _knn3_bruteforce(pts), rtol=1e-4, atol=1e-6)
    # and exactly the oracle's value: the same three float distances, summed alike
    np.testing.assert_array_equal(got, Oracle("restatement").knn3_mean_dist(pts))


@pytest.mark.parametrize("n", [1, 2, 3, 4, 33, 100_000])
def test_gpu_knn_sizes(n):
    pts = np.random.default_rng(n).uniform(-3, 3, (n, 3)).astype(np.float32)
    np.testing.assert_array_equal(_core._gpu_knn3_mean_dist(pts), Oracle("restatement").knn3_mean_dist(pts))


def test_gpu_knn_counts_its_distance_evaluations():
    """33 points make two boxes of the Morton order, and with no neighbours found yet
    every box passes its bounds test: box 0's 32 queries and box 1's single query each
    compute 32 distances per box, 2 x (32 + 1) x 32 in all."""
    pts = torch.from_numpy(np.random.default_rng(4).uniform(-1, 1, (33, 3)).astype(np.float32)).cuda()
    ctx = Context()
    ctx.knn3_mean_dist(pts)
    assert int(ctx.frame("knn_evals").view(torch.int64)[0]) == 2 * 33 * 32


def _f32_ulps(a, b):
    ia = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    ib = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    ia = np.where(ia < 0, -(2 ** 31) - ia, ia)
    ib = np.where(ib < 0, -(2 ** 31) - ib, ib)
    return np.abs(ia - ib)


def test_gpu_init_gaussians():
    rng = np.random.default_rng(11)
    pts = rng.uniform(-2, 2, (20_000, 3)).astype(np.float32)
    rgb = rng.integers(0, 256, (20_000, 3)).astype(np.uint8)
    logit = float(np.log(0.1 / 0.9))
    s, q, d, o = Oracle("restatement").init_gaussians(pts, rgb, 42, logit)
    p = Context().init_gaussians(torch.from_numpy(pts).cuda(), torch.from_numpy(rgb), 42, logit)
    # log / sin / cos in double, rounded once: within 2 ulps of glibc's float functions
    assert _f32_ulps(p.scales.cpu().numpy(), s).max() <= 2
    assert _f32_ulps(p.quats.cpu().numpy(), q).max() <= 2
    assert np.array_equal(p.features_dc.cpu().numpy(), d)
    assert np.array_equal(p.opacities.cpu().numpy(), o)


def _densify_inputs(n, cap, seed):
    rng = np.random.default_rng(seed)
    g = scenes.random_gaussians(n, seed, log_scale_mean=-4.0, log_scale_std=1.5)
    strides = [3, 3, 4, 3, 45, 1]
    bufs = [np.pad(a.reshape(n, s), ((0, cap - n), (0, 0))).astype(np.float32) for a, s in zip(g.arrays(), strides)]
    m1 = [rng.random((cap, s)).astype(np.float32) for s in strides]
    m2 = [rng.random((cap, s)).astype(np.float32) for s in strides]
    stats = {"vis": rng.integers(0, 4, n).astype(np.float32), "gn": (rng.random(n) * 2e-3).astype(np.float32),
             "ms": (rng.random(n) * 0.3).astype(np.float32)}
    return bufs, m1, m2, stats


@pytest.mark.parametrize("n,check_screen,check_huge", [(2000, 1, 1), (2000, 0, 1), (2000, 1, 0), (50_000, 1, 1),
                                                        (1, 1, 1)])
def test_gpu_densify_matches_oracle(n, check_screen, check_huge):
    cap = 3 * n + 7
    bufs, m1, m2, stats = _densify_inputs(n, cap, 40 + n)
    ob, o1, o2 = [b.copy() for b in bufs], [b.copy() for b in m1], [b.copy() for b in m2]
    new_o = Oracle("restatement").densify(n, cap, ob, o1, o2, stats, 60.0, 777, check_screen=check_screen,
                                          check_huge=check_huge)
    tb = [torch.from_numpy(b).cuda() for b in bufs]
    t1 = [torch.from_numpy(b).cuda() for b in m1]
    t2 = [torch.from_numpy(b).cuda() for b in m2]
    st = [torch.from_numpy(stats[k]).cuda() for k in ("gn", "vis", "ms")]
    new_n = Context().densify(n, tb, t1, t2, st[0], st[1], st[2], 60.0, 777, check_screen=bool(check_screen),
                              check_huge=bool(check_huge))
    assert new_n == new_o
    for g in range(6):
        got, ref = tb[g].cpu().numpy()[:new_n], ob[g][:new_n]
        # split offsets come from log / cos / sin (double, rounded once) and exp: a
        # one-ulp offset difference, absolute, on a child mean that may be near zero
        np.testing.assert_allclose(got, ref, rtol=1e-6, atol=1e-7, err_msg=str(g))
        assert (_f32_ulps(got, ref) > 0).any(axis=1).sum() <= max(4, new_n // 200), g
        assert np.array_equal(t1[g].cpu().numpy()[:new_n], o1[g][:new_n]), g
        assert np.array_equal(t2[g].cpu().numpy()[:new_n], o2[g][:new_n]), g


def _split_and_clone_inputs(n, cap, seed):
    """Small Gaussians (world scale below size_thresh) that are large on screen and
    have high gradients: each one is both split and cloned, 4 n rows in all."""
    bufs, m1, m2, stats = _densify_inputs(n, cap, seed)
    bufs[1][:n] = np.log(0.004)  # every scale small: cloned
    stats["vis"][:] = 2.0
    stats["gn"][:] = 1e-3      # (gn / vis) * half_max_dim > 2e-4: high gradient
    stats["ms"][:] = 0.1       # > screen_thresh 0.05: split on screen size
    return bufs, m1, m2, stats


def test_gpu_densify_split_and_clone_needs_4n_rows():
    n = 3000
    cap = 4 * n
    bufs, m1, m2, stats = _split_and_clone_inputs(n, cap, 9)
    ob, o1, o2 = [b.copy() for b in bufs], [b.copy() for b in m1], [b.copy() for b in m2]
    new_o = Oracle("restatement").densify(n, cap, ob, o1, o2, stats, 60.0, 5, check_huge=0)
    tb = [torch.from_numpy(b).cuda() for b in bufs]
    t1 = [torch.from_numpy(b).cuda() for b in m1]
    t2 = [torch.from_numpy(b).cuda() for b in m2]
    st = [torch.from_numpy(stats[k]).cuda() for k in ("gn", "vis", "ms")]
    new_n = Context().densify(n, tb, t1, t2, st[0], st[1], st[2], 60.0, 5, check_huge=False)
    assert new_n == new_o and new_n > 3 * n - n // 2  # the parents are culled, children and clones kept
    for g in range(6):
        np.testing.assert_allclose(tb[g].cpu().numpy()[:new_n], ob[g][:new_n], rtol=1e-6, atol=1e-7)
    # the same Gaussians against 3 n rows: refused, nothing written
    bufs, m1, m2, stats = _split_and_clone_inputs(n, 3 * n, 9)
    tb = [torch.from_numpy(b).cuda() for b in bufs]
    t1 = [torch.from_numpy(b).cuda() for b in m1]
    t2 = [torch.from_numpy(b).cuda() for b in m2]
    st = [torch.from_numpy(stats[k]).cuda() for k in ("gn", "vis", "ms")]
    with pytest.raises(RuntimeError, match="4 N rows"):
        Context().densify(n, tb, t1, t2, st[0], st[1], st[2], 60.0, 5, check_huge=False)
    for t, b in zip(tb + t1 + t2, bufs + m1 + m2):
        assert np.array_equal(t.cpu().numpy(), b)


def test_gpu_densify_capacity_error():
    n = 10
    bufs = [torch.zeros((25, s), device="cuda") for s in (3, 3, 4, 3, 45, 1)]
    with pytest.raises(RuntimeError, match="exceeds buf_capacity"):
        Context().densify(n, bufs, bufs, bufs, bufs[5][:, 0], bufs[5][:, 0], bufs[5][:, 0], 10.0, 1)


def test_gpu_opacity_reset():
    rng = np.random.default_rng(1)
    o = rng.normal(0, 2, 1000).astype(np.float32)
    a = rng.random(1000).astype(np.float32)
    b = rng.random(1000).astype(np.float32)
    oo, aa, bb = o.copy(), a.copy(), b.copy()
    Oracle("restatement").opacity_reset(oo, aa, bb, 1000, -1.3862943611198906)
    to, ta, tb = (torch.from_numpy(x).cuda() for x in (o, a, b))
    Context().opacity_reset(to, ta, tb, 1000)
    assert np.array_equal(to.cpu().numpy(), oo)
    assert np.array_equal(ta.cpu().numpy(), aa) and np.array_equal(tb.cpu().numpy(), bb)


def test_rasterizer_exponential_matches_double_exp():
    """The rasterizers' exponential (Tang's table-driven method in double precision,
    rounded once to float) against CUDA's double exp rounded once (the rounding the
    kernels used before, which agrees with glibc's expf on 99.98 % of floats): over
    every float in [-1, 0] and 16 M random ones in [-5.55, -1], equal except where
    exp(x) sits within ~1e-15 of a float rounding boundary -- then by one ulp."""
    import ctypes as C
    from msplat_street_b200 import _lib
    ctx = Context()
    one = int(np.float32(1.0).view(np.int32))
    chunks = [torch.arange(s, min(s + (1 << 26), one + 1), dtype=torch.int32, device="cuda").view(torch.float32).neg()
              for s in range(0, one + 1, 1 << 26)]
    chunks.append(torch.from_numpy(np.random.default_rng(0).uniform(-5.55, -1.0, 16 << 20).astype(np.float32)).cuda())
    worst, differ, total = 0, 0, 0
    for xt in chunks:
        got = torch.empty_like(xt)
        _lib.check(_lib.lib().msplat_cuda_rasterizer_exp(ctx.handle, C.c_void_p(xt.data_ptr()), xt.numel(),
                                                          C.c_void_p(got.data_ptr())))
        ref = torch.exp(xt.double()).float()
        diff = (got.view(torch.int32).long() - ref.view(torch.int32).long()).abs()
        worst = max(worst, int(diff.max()))
        differ += int((diff > 0).sum())
        total += xt.numel()
    assert worst <= 1
    assert differ <= max(4, total // 10_000_000), (differ, total)
