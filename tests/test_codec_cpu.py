"""The 16-bit fixed-point codec of the solver's spinors, checked on the CPU.

The kernels store a component v in [-32768, 32767] offset-binary, u = v + 32768,
and never use an integer<->float conversion instruction:
- decode places u in the low mantissa bits of 2^23 (bit pattern 0x4B000000 | u)
  and subtracts 2^23 + 32768, exactly;
- encode adds 2^23 + 32768 to the scaled value in FP32, which rounds to the
  nearest integer (ties to even) and leaves u in the low 16 bits.
These identities are checked here for every 16-bit pattern (decode) and for
every FP32 value a kernel can encode at and around the half-integers (encode),
with numpy's IEEE FP32 arithmetic standing in for the GPU's."""
import numpy as np

OFFSET = np.float32(8421376.0)  # 2^23 + 32768


def decode(u):
    bits = np.uint32(0x4B000000) | u.astype(np.uint32)
    return bits.view(np.float32) - OFFSET


def encode(y):
    t = (y.astype(np.float32) + OFFSET).astype(np.float32)
    return t.view(np.uint32) & np.uint32(0xFFFF)


def test_decode_is_exact_for_every_pattern():
    u = np.arange(65536, dtype=np.uint32)
    v = decode(u)
    assert v.dtype == np.float32
    assert np.array_equal(v.astype(np.int64), u.astype(np.int64) - 32768)


def test_encode_rounds_to_nearest_even_and_offsets():
    # every integer, every half-integer (ties) and values just off them
    k = np.arange(-32767, 32768, dtype=np.float64)
    ys = [k, k + 0.5, k - 0.5, k + 0.25, k - 0.25, k + 0.4999, k - 0.4999]
    y = np.concatenate(ys)
    y = y[np.abs(y) <= 32767.49].astype(np.float32)
    got = encode(y)
    want = (np.rint(y.astype(np.float64)).astype(np.int64) + 32768).astype(np.uint32)  # rint: ties to even
    assert np.array_equal(got, want)


def test_round_trip_of_scaled_components():
    """The kernels encode x * (32767 / max) and decode u * (max / 32767): the
    round trip is within half a step (plus the FP32 roundings of the scaling,
    about 1% of a step) of the site's largest component."""
    rng = np.random.default_rng(5)
    x = rng.standard_normal((1000, 24)).astype(np.float32)
    mx = np.abs(x).max(axis=1, keepdims=True)
    sc = np.float32(32767.0) / mx
    u = encode((x * sc).astype(np.float32))
    back = decode(u) * (mx * np.float32(1.0 / 32767.0))
    err = np.abs(back - x) / mx
    assert err.max() <= 0.51 / 32767
    # the largest component maps to +-32767 exactly
    assert np.all(np.abs(decode(u)).max(axis=1) == 32767)
