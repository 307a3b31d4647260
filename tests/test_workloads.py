"""Benchmark workload definitions (mixed batch, GBR 4:4:4 + alpha): every
configuration the mixed-batch generator draws is valid, and the slice
corruption used for the concealment check is seeded and touches payload bytes
only. CPU-only; the GPU side is exercised by bench.py and test_gpu_parity."""
from topos_codec_b200 import binding as B, synth, workloads as WL


def test_mixed_specs_are_valid_and_seeded(oracle):
    specs = WL.mixed_specs(64, seed=0)
    assert specs == WL.mixed_specs(64, seed=0)
    assert {(w, h) for w, h, _, _ in specs} <= set(WL.MIXED_RES)
    assert {t for _, _, t, _ in specs} <= set(WL.MIXED_TIERS)
    assert all(2 <= q <= 16 for _, _, _, q in specs)
    for w, h, t, q in specs:
        assert oracle.validate(WL.mixed_config(w, h, t, q)) == B.TC_OK, (w, h, t, q)
    assert oracle.validate(WL.gbr_config()) == B.TC_OK


def test_corrupt_slices_payload_only(oracle):
    cfg = WL.gbr_config(96, 64)
    cfg.slice_rows = 2
    pkts = [oracle.encode(cfg, synth.make_frame_np(96, 64, seed=s, bit_depth=12, pixel_format=2, limited=False,
                                                   alpha=True, sigma=12)) for s in range(3)]
    bad = WL.corrupt_slices(pkts, 0.1, seed=5)
    assert bad == WL.corrupt_slices(pkts, 0.1, seed=5)
    nspans = sum(len(WL.slice_spans(p)) for p in pkts)
    changed = 0
    for p, q in zip(pkts, bad):
        assert len(p) == len(q) and p[:53] == q[:53]
        for ho, po, size in WL.slice_spans(p):
            assert p[ho:po] == q[ho:po]  # slice headers intact
            changed += p[po:po + size] != q[po:po + size]
    assert changed == max(1, round(0.1 * nspans))
    # the product of the damage decodes with concealed slices, as the reference does
    d = oracle.decode_status(bad[0])
    assert d.status in (B.TC_OK, B.TC_WARN_CONCEALED)


def test_invariant_division_method():
    """The forward quantiser divides by a plane's fixed steps with the
    Granlund-Montgomery round-up multiply (magic m, shifts s1/s2, computed on
    the host for each step): exact for every 32-bit numerator, checked here
    on the method's edge numerators and on random ones for steps 1..2^32-1."""
    import numpy as np

    def magic(d):
        l = 0
        while l < 32 and (1 << l) < d:
            l += 1
        m = ((1 << 32) * ((1 << l) - d)) // d + 1
        return m, (1 if l else 0), (l - 1 if l else 0)

    rng = np.random.default_rng(5)
    ds = list(range(1, 600)) + [int(x) for x in rng.integers(1, 2 ** 32, 400, dtype=np.uint64)]
    ds += [2 ** k for k in range(32)] + [2 ** k + 1 for k in range(1, 32)] + [2 ** k - 1 for k in range(2, 33)]
    for d in ds:
        m, s1, s2 = magic(d)
        assert 0 < m < 2 ** 32
        ns = np.concatenate([rng.integers(0, 2 ** 32, 2000, dtype=np.uint64),
                             np.array([0, 1, d - 1, d, d + 1, 2 ** 32 - 1, 2 ** 32 - d, 2 ** 31, 2 ** 31 - 1],
                                      dtype=np.uint64) % (2 ** 32)])
        t = (ns * np.uint64(m)) >> np.uint64(32)
        q = (t + ((ns - t) >> np.uint64(s1))) >> np.uint64(s2)
        assert np.array_equal(q, ns // np.uint64(d)), d


def test_double_precision_inverse_transform_is_exact():
    """Reconstruction of planes up to 12 bits runs the two 8-point passes of
    the inverse transform in double precision: with coefficients clamped to
    +-2^25 every product and partial sum is an integer below 2^51, so the
    result equals the 64-bit integer passes, including the sign-split
    rounding shift; checked here on random and extreme coefficient blocks."""
    import numpy as np
    M = np.array([13, 13, 13, 13, 13, 13, 13, 13, 13, 11, 7, 1, -1, -7, -11, -13,
                  12, 5, -5, -12, -12, -5, 5, 12, 11, -4, -13, -8, 8, 13, 4, -11,
                  9, -9, -9, 9, 9, -9, -9, 9, 8, -13, 4, 11, -11, -4, 13, -8,
                  5, -12, 12, -5, -5, 12, -12, 5, 1, -7, 11, -13, 13, -11, 7, -1], dtype=np.int64).reshape(8, 8)
    W = np.array([2350, 4672, 4699, 4293, 4902, 4293, 4699, 4672, 4672, 9288, 9343, 8535, 9747, 8535, 9343, 9288,
                  4699, 9343, 9399, 8586, 9805, 8586, 9399, 9343, 4293, 8535, 8586, 7843, 8957, 7843, 8586, 8535,
                  4902, 9747, 9805, 8957, 10228, 8957, 9805, 9747, 4293, 8535, 8586, 7843, 8957, 7843, 8586, 8535,
                  4699, 9343, 9399, 8586, 9805, 8586, 9399, 9343, 4672, 9288, 9343, 8535, 9747, 8535, 9343, 9288],
                 dtype=np.int64).reshape(8, 8)

    def rs_int(v):
        return np.where(v >= 0, (v + (1 << 31)) >> 32, -((-v + (1 << 31)) >> 32))

    def rs_f64(v):
        r = np.floor((np.abs(v) + 2147483648.0) * 2.0 ** -32)
        return np.where(v >= 0.0, r, -r).astype(np.int64)

    rng = np.random.default_rng(11)
    lim = 1 << 25
    blocks = [rng.integers(-lim, lim + 1, (8, 8)) for _ in range(3000)]
    blocks += [np.full((8, 8), lim), np.full((8, 8), -lim), np.where(M > 0, lim, -lim), np.where(M.T > 0, -lim, lim)]
    blocks += [rng.choice([-lim, lim], (8, 8)) for _ in range(500)]
    blocks += [rng.integers(-40, 41, (8, 8)) for _ in range(500)]
    for c in blocks:
        G = c.astype(np.int64) * W                 # G = c (.) W
        B = G @ M                                   # B[u][x] = sum_v G[u][v] M[v][x]
        xi = rs_int(M.T @ B)                        # xhat[y][x] = rs(sum_u M[u][y] B[u][x])
        Gd = c.astype(np.float64) * W.astype(np.float64)
        Bd = Gd @ M.astype(np.float64)
        assert np.abs(Bd).max() < 2.0 ** 51
        xd = rs_f64(M.T.astype(np.float64) @ Bd)
        assert np.array_equal(xi, xd)
