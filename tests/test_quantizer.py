"""Int8Quantizer on the GPU (src/quantize.rs:45-96) against the oracle's
restatement: shift, scale, codes and clipped counts bit-exact."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FAISS = (112.0, 1.0, True)


def _cal(emb, t):
    return emb.Calibration(target_peak=t[0], quantile=t[1], power_of_two=t[2])


@pytest.fixture(scope="module")
def qa(emb):
    a = emb.B200Assigner(0)
    yield a
    a.close()


def test_reference_golden(emb, qa):
    # src/quantize.rs:102-116
    sample = np.array([15.0, -3.0, 5.0, -3.0, 10.0, -2.0, 10.0, -4.0], np.float32)
    q = emb.Int8Quantizer.fit(sample, 2, emb.Calibration.faiss(), assigner=qa)
    assert q.shift.tolist() == [10.0, -3.0]
    assert q.scale == 16.0
    codes = q.encode(sample, assigner=qa)
    assert codes.tolist() == [80, 0, -80, 0, 0, 16, 0, -16]
    back = q.decode(codes.astype(np.float32), assigner=qa)
    assert np.array_equal(back, sample)
    assert q.decode_sqdist(256.0) == 1.0
    assert q.encode(np.array([1000.0, -3.0], np.float32), assigner=qa).tolist() == [127, 0]
    assert q.clipped_fraction(np.array([1000.0, -3.0], np.float32), assigner=qa) == 0.5


@pytest.mark.parametrize("n,d", [(1, 1), (7, 3), (1000, 1), (4097, 96), (3000, 130), (517, 512), (20000, 33)])
@pytest.mark.parametrize("cal", [FAISS, (127.0, 0.9999, False), (127.0, 0.5, False), (127.0, 0.0, False),
                                 (100.0, 0.37, True)])
def test_fit_encode_match_oracle(emb, orc, qa, n, d, cal):
    rng = np.random.default_rng(n * 1000 + d)
    # heavy-tailed, offset per dimension, with repeated values (ties at the quantile)
    x = (rng.standard_t(3.0, (n, d)) * rng.uniform(0.1, 3.0, d) + rng.normal(0, 5, d)).astype(np.float32)
    x[rng.random((n, d)) < 0.05] = 1.5
    q = emb.Int8Quantizer.fit(x, d, _cal(emb, cal), assigner=qa)
    shift, scale = orc.quantizer_fit(x, *cal)
    assert np.array_equal(q.shift.view(np.uint32), shift.view(np.uint32))
    assert np.float32(q.scale).view(np.uint32) == np.float32(scale).view(np.uint32), (q.scale, scale)
    codes = q.encode(x, assigner=qa)
    assert np.array_equal(codes, orc.quantizer_encode(x, shift, scale))
    assert q.clipped_fraction(x, assigner=qa) == orc.quantizer_clipped(x, shift, scale) / x.size


def test_fit_on_device_rows_and_resident_rows(emb, orc):
    import torch

    rng = np.random.default_rng(11)
    x = rng.normal(0.3, 1.0, (5000, 64)).astype(np.float32)
    a = emb.B200Assigner(0)
    cal = emb.Calibration.clipped(0.999)
    ref_shift, ref_scale = orc.quantizer_fit(x, 127.0, 0.999, False)
    xd = torch.from_numpy(x).cuda()
    shift = np.empty(64, np.float32)
    scale = ctypes.c_float()
    c = cal._c()
    a._check(emb.lib().emb200_quantizer_fit_device(a._h, ctypes.c_void_p(xd.data_ptr()), 5000, 64, ctypes.byref(c),
                                                   shift.ctypes.data_as(ctypes.c_void_p), ctypes.byref(scale)))
    assert np.array_equal(shift, ref_shift) and np.float32(scale.value) == np.float32(ref_scale)
    codes_d = torch.empty((5000, 64), dtype=torch.int8, device="cuda")
    clipped = ctypes.c_uint64()
    a._check(emb.lib().emb200_quantizer_encode_device(
        a._h, ctypes.c_void_p(xd.data_ptr()), 5000, 64, shift.ctypes.data_as(ctypes.c_void_p), scale.value,
        ctypes.c_void_p(codes_d.data_ptr()), ctypes.byref(clipped), None))
    ref_codes = orc.quantizer_encode(x, ref_shift, ref_scale)
    assert np.array_equal(codes_d.cpu().numpy(), ref_codes)
    assert clipped.value == orc.quantizer_clipped(x, ref_shift, ref_scale)
    # resident rows: fit, quantize in place, then the int8 search sees the codes
    a.load_rows(x)
    q = emb.Int8Quantizer.fit_resident(a, cal)
    assert np.array_equal(q.shift, ref_shift) and q.scale == np.float32(ref_scale)
    assert q.quantize_resident(a) == clipped.value
    cent = ref_codes[:40].astype(np.float32)
    a.set_options(centroid_bits=8)
    a.set_centroids(cent)
    lab_r, dist_r = a.assign_resident()
    lab_h, dist_h = a.assign(ref_codes)
    assert np.array_equal(lab_r, lab_h) and np.array_equal(dist_r.view(np.uint32), dist_h.view(np.uint32))
    a.close()


def test_encode_rounding_clamp_and_non_finite(emb, orc, qa):
    d = 5
    shift = np.zeros(d, np.float32)
    q = emb.Int8Quantizer(d, shift, 1.0)
    v = np.array([0.5, -0.5, 1.5, -1.5, 2.4999998, 126.5, 127.49999, 127.5, -128.5, -128.50002, 300.0, -300.0,
                  np.inf, -np.inf, np.nan, 0.49999997, -0.0, 1e30, -1e-30, 3.5], np.float32)
    codes = q.encode(v.reshape(-1, d), assigner=qa).ravel()
    ref = orc.quantizer_encode(v.reshape(-1, d), shift, 1.0).ravel()
    assert codes.tolist() == ref.tolist()
    assert codes[:5].tolist() == [1, -1, 2, -2, 2]  # half away from zero
    assert codes[14] == 0  # NaN -> 0
    assert q.clipped_fraction(v.reshape(-1, d), assigner=qa) == orc.quantizer_clipped(v.reshape(-1, d), shift,
                                                                                      1.0) / v.size


def test_fit_peak_with_inf_and_constant_rows(emb, orc, qa):
    # A constant sample has peak 0, so scale 1 (src/quantize.rs:57). One infinite
    # value makes its dimension's shift inf and the magnitudes there inf or NaN
    # (inf - inf); NaN is the largest under f32::total_cmp, so the peak is NaN and
    # the scale 1 again.
    x = np.full((100, 4), 2.5, np.float32)
    q = emb.Int8Quantizer.fit(x, 4, emb.Calibration.faiss(), assigner=qa)
    assert q.scale == 1.0 and np.all(q.shift == 2.5)
    x[3, 1] = np.inf
    q = emb.Int8Quantizer.fit(x, 4, emb.Calibration.faiss(), assigner=qa)
    shift, scale = orc.quantizer_fit(x)
    assert np.array_equal(q.shift, shift, equal_nan=True) and q.scale == np.float32(scale) == 1.0


def test_large_unit_norm_rows(emb, orc, qa):
    # 1M x 128 unit-norm rows (the shape of the 1M x 128 assign workload) at both
    # calibrations of examples/int8.rs:46.
    x = emb.datasets.embeddings(1_000_000, 128, latent=32, seed=2)
    for cal in (FAISS, (127.0, 0.9999, False)):
        q = emb.Int8Quantizer.fit(x, 128, _cal(emb, cal), assigner=qa)
        shift, scale = orc.quantizer_fit(x, *cal)
        assert np.array_equal(q.shift, shift) and q.scale == np.float32(scale)
        codes = q.encode(x, assigner=qa)
        assert np.array_equal(codes, orc.quantizer_encode(x, shift, scale))


def test_quantizer_errors(emb, qa):
    lib = emb.lib()
    scale = ctypes.c_float()
    shift = np.zeros(4, np.float32)
    cal = emb.Calibration.faiss()._c()
    x = np.ones((3, 4), np.float32)
    # an empty sample (src/quantize.rs:47 asserts n > 0), a null sample
    assert lib.emb200_quantizer_fit(qa._h, x.ctypes.data_as(ctypes.c_void_p), 0, 4, ctypes.byref(cal),
                                    shift.ctypes.data_as(ctypes.c_void_p), ctypes.byref(scale)) == -1
    assert lib.emb200_quantizer_fit(qa._h, None, 3, 4, ctypes.byref(cal), shift.ctypes.data_as(ctypes.c_void_p),
                                    ctypes.byref(scale)) == -1
    # device rows must be 16-byte aligned
    import torch

    xd = torch.ones(64, dtype=torch.float32, device="cuda")
    assert lib.emb200_quantizer_fit_device(qa._h, ctypes.c_void_p(xd.data_ptr() + 4), 3, 4, ctypes.byref(cal),
                                           shift.ctypes.data_as(ctypes.c_void_p), ctypes.byref(scale)) == -1
    assert "aligned" in lib.emb200_last_error(qa._h).decode()
    # the resident rows must be f32
    a = emb.B200Assigner(0)
    a.load_rows(np.zeros((8, 4), np.int8))
    with pytest.raises(emb.EngineError):
        emb.Int8Quantizer.fit_resident(a, emb.Calibration.faiss())
    with pytest.raises(emb.EngineError):
        emb.Int8Quantizer(4, shift, 1.0).quantize_resident(a)
    a.close()
