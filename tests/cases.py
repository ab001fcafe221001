"""Seeded parity cases shared by the GPU tests and the golden-fixture generator."""
import numpy as np

from chaincompressor_b200 import workloads as W


def case(name):
    """-> (points (N, D), eb, p, threshold, kwargs)"""
    if name == "column":
        pts = W.column()
        return pts, W.eb_for(pts, 1e-3), 4, 2, {}
    if name == "column_qb11":
        pts = W.column()
        return pts, float(np.max(pts.max(0).astype(np.float64) - pts.min(0))) / (2 ** 11 - 2), 256, 4, {}
    if name == "blobs200k":
        pts = W.blobs(200_000, 11)
        return pts, W.eb_for(pts, 1e-3), 4, 2, {}
    if name == "blobs_clipped":
        pts = W.blobs(100_000, 12, clip=True)
        return pts, W.eb_for(pts, 1e-3), 4, 2, {}
    if name == "traj_f64_e4_p1":
        pts = W.trajectory(0, 60_000)
        return pts, W.eb_for(pts, 1e-4), 1, 2, {}
    if name == "traj_f64_e2":
        pts = W.trajectory(3, 50_000)
        return pts, W.eb_for(pts, 1e-2), 4, 2, {}
    if name == "uniform_p64_t25":
        pts = W.uniform(30_000, 5)
        return pts, W.eb_for(pts, 1e-4), 64, 25, {}
    if name == "single_point":
        return np.array([[1.5, -2.0, 3.25]], np.float64), 0.01, 4, 2, {}
    if name == "one_block":
        rng = np.random.default_rng(9)
        pts = rng.uniform(0, 1, size=(5000, 3)).astype(np.float32)
        return pts, 0.01, 1 << 20, 0, {}
    if name == "long_chain":
        # a few blocks holding almost every point: level-1 chains of tens of thousands of
        # links, longer than the decoder's one-pass resolution follows (exercises the
        # pointer-jumping rounds); block coordinates far from the frame minimum make
        # chaining pay off
        rng = np.random.default_rng(14)
        pts = rng.uniform(1000.0, 1001.2, size=(300_000, 3)).astype(np.float32)
        pts[0] = 0.0
        return pts, 0.01, 64, 2, {}
    if name == "p1_big_threshold":
        pts = W.column(20_000, 3)
        return pts, W.eb_for(pts, 1e-3), 1, 1000, {}
    if name == "neg_threshold":
        pts = W.column(20_000, 4)
        return pts, W.eb_for(pts, 1e-3), 2, -5, {}
    if name == "dims1":
        rng = np.random.default_rng(10)
        return rng.normal(0, 3, size=(40_000, 1)), 1e-3, 8, 1, {}
    if name == "dims2":
        rng = np.random.default_rng(11)
        return rng.normal(0, 3, size=(40_000, 2)).astype(np.float32), 1e-3, 4, 2, {}
    if name == "dims4":
        rng = np.random.default_rng(12)
        return rng.uniform(-5, 5, size=(20_000, 4)), 1e-2, 4, 2, {}
    if name == "dims6":
        # more than four dimensions: the statistics kernel that reads D at run time
        rng = np.random.default_rng(17)
        return rng.uniform(-5, 5, size=(20_000, 6)).astype(np.float32), 1e-2, 4, 2, {}
    if name == "big_q":
        # quantized values between 2^31 and 2^32 (about 3.3e9 steps per axis; p = 4 gives
        # 30-bit block coordinates and 90-bit block keys)
        rng = np.random.default_rng(18)
        return rng.uniform(0, 1, size=(20_000, 3)), 1.5e-10, 4, 2, {}
    if name == "no_l1":
        pts = W.column(20_000, 5)
        return pts, W.eb_for(pts, 1e-3), 4, 2, {"l1": False}
    if name == "no_l2":
        pts = W.column(20_000, 6)
        return pts, W.eb_for(pts, 1e-3), 4, 2, {"l2": False}
    if name == "no_bl":
        pts = W.column(20_000, 7)
        return pts, W.eb_for(pts, 1e-3), 16, 2, {"bl": False}
    if name == "big_values_tagged":
        # wide jumps and large block ids push alphabets past 2^18 (tagged/fixed codings)
        rng = np.random.default_rng(13)
        pts = rng.uniform(0, 1, size=(300_000, 2))
        return pts, 1e-7, 2, -40, {}
    if name == "wide_jump":
        # a chain distance above 2^18: point 0 and point n-1 share a block, all others
        # are alone (idrel alphabet too large for raw rANS)
        n = 400_000
        pts = np.arange(n, dtype=np.float64).reshape(n, 1)
        pts[-1, 0] = 1.0
        return pts, 0.5, 1, -30, {}
    if name == "many_corrections":
        # half the points on the far corner of the box, where the float64 reconstruction
        # of every coordinate misses the bound: more than 2^20 exact corrections
        rng = np.random.default_rng(15)
        pts = rng.uniform(0, 1, size=(1 << 20, 3))
        pts[: 1 << 19] = 1.0
        pts[-1] = 0.0
        return pts, 0.1, 4, 2, {}
    if name == "wide_key":
        # three dimensions of 25 block-coordinate bits (p = 1): 75-bit block keys; 2,000
        # distinct blocks of about 30 points each, shuffled, so level 1 still chains
        rng = np.random.default_rng(16)
        blocks = rng.integers(0, 1 << 25, size=(2000, 3)).astype(np.float64)
        pts = blocks[rng.integers(0, 2000, size=60_000)] + 0.5
        pts[0] = 0.5
        return pts, 0.5, 1, 2, {}
    if name == "negative_zero":
        pts = np.array([[0.0, -0.0], [-0.0, 0.0], [1.0, 2.0], [0.5, -0.0]], np.float64)
        return pts, 0.05, 2, 0, {}
    raise KeyError(name)


GPU_CASES = ["column", "column_qb11", "blobs200k", "blobs_clipped", "traj_f64_e4_p1", "traj_f64_e2",
             "uniform_p64_t25", "single_point", "one_block", "long_chain", "p1_big_threshold", "neg_threshold", "dims1", "dims2",
             "dims4", "dims6", "big_q", "no_l1", "no_l2", "no_bl", "big_values_tagged", "wide_jump", "negative_zero", "many_corrections", "wide_key"]
