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
