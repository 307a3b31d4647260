"""Size-targeted encode (tc_frame_encode_sized) through the C-ABI against the
reference library built from its sources (oracle/_ref): for the same call
sequence the status, chosen qp, packet bytes, stats and probe-encode count
agree, in the strict (default), linear and r6 search modes, including the
cross-call qp hint, qp ranges above 63, unreachable and trivially met
targets, a too-small output buffer and a 4:4:4 + alpha frame."""
import numpy as np
import pytest

from topos_codec_b200 import binding as B, synth

pytestmark = pytest.mark.gpu


def _sized(codec, cfg, planes, target, qp_min, qp_max, cap=None):
    lib = codec._lib
    it0 = lib.tc_dev_sized_iters()
    rc, pkt, st, qp, out = codec.encode_sized_status(cfg, planes, target, qp_min, qp_max, cap)
    iters = lib.tc_dev_sized_iters() - it0
    untouched = bool(np.all(out == 0xA5)) if rc != 0 else None
    return {"rc": rc, "qp": qp, "pkt": pkt, "size": st.packet_size, "qp_base": st.qp_base,
            "color": st.color_payload_bytes, "alpha": st.alpha_payload_bytes, "slices": st.slice_count,
            "iters": iters, "untouched": untouched}


def _both(product, reference, cfg, planes, target, qp_min, qp_max, cap=None):
    a = _sized(product, cfg, planes, target, qp_min, qp_max, cap)
    b = _sized(reference, cfg, planes, target, qp_min, qp_max, cap)
    assert a == b, {k: (a[k], b[k]) for k in a if a[k] != b[k] and k != "pkt"}
    return a


@pytest.fixture(scope="module")
def libs(product, reference):
    yield product, reference
    for c in (product, reference):
        c._lib.tc_dev_set_sized_mode(0)
        c._lib.tc_dev_set_qp_hint(0)


def _frame(w, h, seed, qp=20, **kw):
    planes = synth.make_frame_np(w, h, seed=seed)
    cfg = B.make_config(w, h, qp=qp, qmatrix_id=4, features=1, **kw)
    return cfg, planes


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_sized_modes_vs_reference(libs, mode):
    product, reference = libs
    for c in libs:
        c._lib.tc_dev_set_sized_mode(mode)
        c._lib.tc_dev_set_qp_hint(1)  # a fixed first probe: identical probe sequences
    cfg, planes = _frame(256, 128, seed=90 + mode)
    sizes = {q: len(product.encode(B.make_config(256, 128, qp=q, qmatrix_id=4, features=1), planes))
             for q in (8, 20, 33, 50)}
    for target, lo, hi in [(sizes[33], 0, 63), (sizes[33] - 1, 0, 63), (sizes[20] * 3 // 4, 0, 63),
                           (sizes[8] * 2, 0, 63), (sizes[50] // 3, 10, 40), (64, 0, 40), (sizes[20], 20, 20),
                           (sizes[50], 64, 95), (1, 0, 95), (10 ** 9, 0, 95)]:
        r = _both(product, reference, cfg, planes, target, lo, hi)
        assert r["rc"] == 0 and lo <= r["qp"] <= hi
        # the chosen packet is the plain encode at that qp
        direct = B.make_config(256, 128, qp=r["qp"], qmatrix_id=4, features=1)
        assert r["pkt"] == product.encode(direct, planes)


def test_sized_hint_sequence_vs_reference(libs):
    """Hints on: a run of calls on frames of two sizes with rising and falling
    targets moves both libraries' hint records the same way."""
    product, reference = libs
    for c in libs:
        c._lib.tc_dev_set_sized_mode(0)
        c._lib.tc_dev_set_qp_hint(0)
    cfg_a, pa = _frame(320, 192, seed=7)
    cfg_b, pb = _frame(128, 64, seed=8)
    base = len(product.encode(cfg_a, pa))
    for k, (cfg, planes, target) in enumerate([(cfg_a, pa, base), (cfg_a, pa, base // 2), (cfg_a, pa, base // 5),
                                               (cfg_b, pb, 4000), (cfg_a, pa, base * 2), (cfg_a, pa, base // 3)]):
        r = _both(product, reference, cfg, planes, target, 0, 63)
        assert r["rc"] == 0, k


def test_sized_buffer_too_small_and_alpha_vs_reference(libs):
    product, reference = libs
    for c in libs:
        c._lib.tc_dev_set_sized_mode(0)
        c._lib.tc_dev_set_qp_hint(1)
    cfg, planes = _frame(192, 96, seed=11)
    target = len(product.encode(cfg, planes))
    r = _both(product, reference, cfg, planes, target, 0, 63, cap=64)
    assert r["rc"] == B.TC_ERR_BUFFER_TOO_SMALL and r["untouched"] and r["size"] > 64
    w, h = 160, 96
    planes = synth.make_frame_np(w, h, seed=12, bit_depth=12, pixel_format=2, limited=False, alpha=True, sigma=12)
    cfg = B.make_config(w, h, qp=2, bit_depth=12, pixel_format=2, profile=5, alpha_mode=1, alpha_bit_depth=16,
                        color_range=1)
    full = len(product.encode(cfg, planes))
    for target in (full, full * 2 // 3, full // 3):
        r = _both(product, reference, cfg, planes, target, 0, 63)
        assert r["rc"] == 0 and r["alpha"] > 0


def test_sized_batch_vs_reference_single_calls(libs):
    """tcg_frame_encode_sized_batch: each frame as the reference's single call
    with an empty hint record (hint and its model off), whatever the order;
    searches run side by side on separate contexts."""
    import ctypes
    product, reference = libs
    for c in libs:
        c._lib.tc_dev_set_sized_mode(0)
        c._lib.tc_dev_set_qp_hint(1)
    reference._lib.tc_dev_set_qp_hint_model(1)
    try:
        specs = [(256, 128, 5), (640, 360, 6), (192, 96, 7), (256, 128, 8), (640, 360, 9), (96, 64, 10), (320, 192, 11)]
        cfgs, frames, targets = [], [], []
        for k, (w, h, seed) in enumerate(specs):
            cfg, planes = _frame(w, h, seed=seed, qp=4 + 7 * k)
            full = len(product.encode(cfg, planes))
            cfgs.append(cfg)
            frames.append(planes)
            targets.append([full, full // 2, full * 3, 40][k % 4])
        n = len(specs)
        L = product._lib
        L.tcg_frame_encode_sized_batch.restype = ctypes.c_int32
        caps = [product.packet_bound(c) for c in cfgs]
        bufs = [np.empty(c, np.uint8) for c in caps]
        carr = (B.FrameConfig * n)(*cfgs)
        iarr = (B.FrameInput * n)(*[product._input(f) for f in frames])
        tarr = (ctypes.c_uint32 * n)(*targets)
        qps = (ctypes.c_uint8 * n)()
        optr = (ctypes.c_void_p * n)(*[b.ctypes.data for b in bufs])
        ocap = (ctypes.c_size_t * n)(*caps)
        st = (B.FrameStats * n)()
        rcs = (ctypes.c_int32 * n)()
        it0 = L.tc_dev_sized_iters()
        rc = int(L.tcg_frame_encode_sized_batch(carr, iarr, ctypes.c_uint32(n), tarr, ctypes.c_uint8(0),
                                                ctypes.c_uint8(63), qps, optr, ocap, st, rcs))
        iters = L.tc_dev_sized_iters() - it0
        assert rc == 0 and list(rcs) == [0] * n
        ri0 = reference._lib.tc_dev_sized_iters()
        for i in range(n):
            want = _sized(reference, cfgs[i], frames[i], targets[i], 0, 63)
            assert want["rc"] == 0 and want["qp"] == qps[i], i
            assert bufs[i][: st[i].packet_size].tobytes() == want["pkt"], i
            assert st[i].packet_size == want["size"] and st[i].qp_base == want["qp_base"], i
        assert iters == reference._lib.tc_dev_sized_iters() - ri0
    finally:
        reference._lib.tc_dev_set_qp_hint_model(0)


def test_sized_device_resident_input_equals_host(product, libs):
    """Sample planes in device memory give the host-memory call's packet and qp."""
    import ctypes

    import torch
    for c in libs:
        c._lib.tc_dev_set_sized_mode(0)
        c._lib.tc_dev_set_qp_hint(1)
    cfg, planes = _frame(320, 192, seed=21)
    target = len(product.encode(cfg, planes)) * 2 // 3
    rc, pkt, st, qp, _ = product.encode_sized_status(cfg, planes, target, 0, 63)
    assert rc == 0
    dev = [torch.from_numpy(p.astype(np.int32)).cuda().to(torch.uint16) for p in planes]
    fi = B.FrameInput()
    fi.struct_size, fi.abi_version = ctypes.sizeof(B.FrameInput), 2
    for i, t in enumerate(dev):
        fi.planes[i], fi.strides[i] = t.data_ptr(), t.shape[1]
    cap = product.packet_bound(cfg)
    out = np.empty(cap, np.uint8)
    st2 = B.FrameStats()
    q2 = ctypes.c_uint8()
    rc2 = product._lib.tc_frame_encode_sized(ctypes.byref(cfg), ctypes.byref(fi), target, 0, 63, ctypes.byref(q2),
                                             out.ctypes.data, cap, ctypes.byref(st2))
    assert rc2 == 0 and q2.value == qp and out[: st2.packet_size].tobytes() == pkt
