"""Storage formats of the oracle: binary16 / bfloat16 rounding, the host's
f16 packing of q (lattice.rs:172-189) and stochastic rounding (shader.rs:510-517)."""
import numpy as np

import oracle


def test_f16_round_to_nearest_even_matches_numpy():
    L = oracle.library()
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.standard_normal(2000) * 10.0 ** rng.integers(-9, 5, 2000),
                         [0.0, -0.0, 1e-8, 6e-8, 65504.0, 65520.0, 1e6, 2.0 ** -24, 3 * 2.0 ** -25]]).astype(np.float32)
    for x in xs:
        assert L.orc_f32_to_f16(float(x)) == int(np.float16(x).view(np.uint16)), x
        h = np.float16(x).view(np.uint16)
        back = L.orc_f16_to_f32(int(h))
        assert (np.isnan(back) and np.isnan(np.float32(np.float16(x)))) or back == np.float32(np.float16(x))


def test_bf16_round_to_nearest_even():
    L = oracle.library()
    for x in np.float32([1.0, 1.00390625, 1.01171875, -3.14159, 1e-30, 3e38]):
        b = int(np.array([x], dtype=np.float32).view(np.uint32)[0])
        rounded = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) & 0xFFFF
        assert L.orc_f32_to_bf16(float(x)) == rounded


def test_q_packing_matches_reference_rule():
    L = oracle.library()
    # values in the q range: the reference rounds half up on the magnitude
    for q in np.float32([0.001, 0.5, 0.3333333, 0.9999, 1.0, 0.123456]):
        b = int(np.array([q], dtype=np.float32).view(np.uint32)[0])
        exp = ((b >> 23) & 0xFF) - 127 + 15
        man = b & 0x7FFFFF
        h = (exp << 10) | (man >> 13)
        if man & 0x1000:
            h += 1
        assert L.orc_f16_bits_ref(float(q)) == h


def test_stochastic_rounding_is_unbiased_and_bounded():
    L = oracle.library()
    x = np.float32(1234.567)  # f16 ulp at this magnitude is 1.0
    vals = np.array([L.orc_sround16(float(x), k, 7) for k in range(4000)], dtype=np.float32)
    assert np.all(np.abs(vals - x) <= 0.5)
    r = np.array([np.float16(v) for v in vals], dtype=np.float64)
    assert abs(r.mean() - float(x)) < 0.03
    assert L.orc_sround16(1e9, 1, 1) == 65000.0
