"""The 16-bit storage format of MB_PREC_F16C (sign, 3-bit exponent, 12-bit
fraction; kernels.cuh h16c_encode / h16c_decode), restated in numpy: every
code round-trips, conversion rounds to nearest, the spacing is a quarter of
IEEE binary16's for |h| >= 2^-9, and the device codec (set_fields ->
fields through the C ABI) equals this restatement bit for bit.
(Rounding is to nearest within 2^-11 of a code spacing: below 2^-9 the
scaled value passes the FP32 subnormal grid first.)"""
import numpy as np
import pytest

SCALE_UP = np.float32(2.0 ** 117)
SCALE_DN = np.float32(2.0 ** -117)


def decode(u):
    u = np.asarray(u, dtype=np.uint32)
    bits = ((u & 0x7FFF) << 11) | ((u & 0x8000) << 16)
    return bits.astype(np.uint32).view(np.float32) * SCALE_UP


def encode(v):
    v = np.asarray(v, dtype=np.float32)
    with np.errstate(over="ignore", invalid="ignore"):
        b = (v * SCALE_DN).view(np.uint32).astype(np.uint64)
    mag = b & 0x7FFFFFFF
    r = np.where(mag >= 0x7F800000, 0x7FFF, (mag + 0x3FF + ((mag >> 11) & 1)) >> 11)
    r = np.minimum(r, 0x7FFF)
    return (r | ((b >> 16) & 0x8000)).astype(np.uint16)


def test_codes_round_trip():
    codes = np.arange(65536, dtype=np.uint32)
    v = decode(codes)
    assert np.all(np.isfinite(v))
    assert np.array_equal(encode(v).astype(np.uint32), codes)
    pos = v[:0x8000]
    assert np.all(np.diff(pos) > 0) and pos[0] == 0.0
    assert float(pos[-1]) < 0.25 and float(pos[-1]) > 0.2499


def test_rounds_to_nearest_and_saturates():
    rng = np.random.default_rng(5)
    v = np.concatenate([rng.uniform(-0.2499, 0.2499, 200000), rng.uniform(-1e-3, 1e-3, 50000)]).astype(np.float32)
    d = decode(encode(v)).astype(np.float64)
    u = encode(v).astype(np.uint32) & 0x7FFF
    up = decode(np.minimum(u + 1, 0x7FFF)).astype(np.float64)
    dn = decode(np.maximum(u.astype(np.int64) - 1, 0).astype(np.uint32)).astype(np.float64)
    a = np.abs(v.astype(np.float64))
    # nearest code; below 2^-9 the scaled value is first rounded to the FP32
    # subnormal grid (2^-11 of a code spacing), so ties may break that far off
    assert np.all(np.abs(a - np.abs(d)) <= (0.5 + 2.0 ** -11) * np.maximum(up - np.abs(d), np.abs(d) - dn))
    big = np.array([0.25, 3.0, np.inf, -np.inf, -0.3, np.nan], dtype=np.float32)
    assert list(encode(big) & 0x7FFF) == [0x7FFF] * 6
    assert list(encode(big)[:5] >> 15) == [0, 0, 0, 1, 1]


def test_spacing_against_binary16():
    for x in (2.0 ** -9, 0.003, 0.0133, 0.05, 0.2):
        c = int(encode(np.float32(x)))
        ours = float(decode(c + 1)) - float(decode(c))
        h = np.float16(x)
        ieee = float(np.nextafter(h, np.float16(1.0))) - float(h)
        assert ours == pytest.approx(ieee / 4, rel=1e-6), x
    assert float(decode(1)) == 2.0 ** -21


@pytest.mark.gpu
def test_device_codec_matches(mb, cuda_device):
    """set_fields -> fields through an F16C context: the stored form of every
    distribution is h16c(float32(f) - w_k), read back as decode + w_k in FP32."""
    import make_ref

    g = mb.geo_init(*make_ref.case("g11")[:2])
    m = mb.MultiBlockLBM(g, "f16c", shift="w")
    m.init()
    A = g.Areas[0]
    n = A.nx * A.ny
    w = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
    rng = np.random.default_rng(11)
    h = np.concatenate([rng.uniform(-0.2, 0.2, 4 * n), rng.uniform(-2e-3, 2e-3, 4 * n),
                        rng.uniform(-2e-6, 2e-6, n)])[: 9 * n].reshape(9, A.ny, A.nx)
    F = w[:, None, None] + h
    m.set_fields(0, F=F)
    got = m.fields(0)["F"]
    w32 = w.astype(np.float32)[:, None, None]
    stored = encode(F.astype(np.float32) - w32)
    want = (decode(stored) + w32).astype(np.float64)
    assert np.array_equal(got, want)
    m.close()
