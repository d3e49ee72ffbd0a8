"""The random stream: published Philox4x32-10 known answers, and the
product's stream against the oracle's (both replace cuRAND's draws of
hpc_code/lib/main.cu:118-120, 140, 144, 282)."""
import numpy as np
import pytest

import pyoracle
from rms_b200 import engine

# Known-answer vectors published with Random123 (Salmon et al., SC'11):
# counter (4 words), key (2 words) -> output (4 words), Philox4x32 with 10 rounds.
KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,want", KAT)
def test_philox_kat_oracle(ctr, key, want):
    assert list(pyoracle.philox4x32_10(ctr, key)) == list(want)


@pytest.mark.parametrize("ctr,key,want", KAT)
def test_philox_kat_product(ctr, key, want):
    assert list(engine.philox4x32_10(ctr, key)) == list(want)


@pytest.mark.parametrize("seed,walker", [(0, 0), (12345, 7), (2**63 + 5, 2**40 + 3)])
def test_streams_match_oracle(seed, walker):
    assert np.array_equal(engine.rng_doubles(seed, walker, 257), pyoracle.stream_doubles(seed, walker, 257))
    assert np.array_equal(engine.rng_floats(seed, walker, 257), pyoracle.stream_floats(seed, walker, 257))


@pytest.mark.parametrize("seed,walker", [(0, 0), (99, 123456), (2**64 - 1, 2**39 + 1)])
def test_split_streams_match_oracle(seed, walker):
    assert np.array_equal(engine.rng_split(seed, walker, 0, 400), pyoracle.split_dir_uniforms(seed, walker, 200))
    for dom in (1, 2):
        assert np.array_equal(engine.rng_split(seed, walker, dom, 101),
                              pyoracle.split_domain_floats(seed, walker, dom, 101))


def test_uniform_maps_open_interval_and_moments():
    d = np.concatenate([engine.rng_doubles(3, w, 2000) for w in range(20)])
    f = np.concatenate([engine.rng_floats(3, w, 2000) for w in range(20)]).astype(np.float64)
    for u in (d, f):
        assert u.min() > 0.0 and u.max() < 1.0
        assert abs(u.mean() - 0.5) < 0.01
        assert abs(u.var() - 1.0 / 12.0) < 0.003


def test_double_map_is_exact():
    # u = (2m+1) 2^-53 with m the top 52 bits of (hi:lo)
    lo, hi = 0x6627E8D5, 0xE169C58D
    m = ((hi << 32) | lo) >> 12
    assert engine.rng_doubles(0, 0, 1)[0] == (2 * m + 1) * 2.0 ** -53


def test_float_map_from_bits_is_exact():
    """The kernels form a uniform float from the word's top 23 bits as
    (1 + k 2^-23) - (1 - 2^-24) (bits of 1.0 or'ed with k); that equals the
    stream's defined value (2k + 1) 2^-24 for every k: the FP32 subtraction
    is exact."""
    k = np.arange(1 << 23, dtype=np.uint32)
    from_bits = (np.uint32(0x3F800000) | k).view(np.float32) - np.float32(1.0 - 2.0 ** -24)
    defined = ((2 * k.astype(np.float64) + 1) * 2.0 ** -24).astype(np.float32)
    assert np.array_equal(from_bits, defined)
    assert np.array_equal(defined.astype(np.float64), (2 * k.astype(np.float64) + 1) * 2.0 ** -24)
    # the direction stream's 21-bit fields: (1 + f 2^-21) - (1 - 2^-22) = (2f + 1) 2^-22
    f = np.arange(1 << 21, dtype=np.uint32)
    from_bits = (np.uint32(0x3F800000) | (f << np.uint32(2))).view(np.float32) - np.float32(1.0 - 2.0 ** -22)
    assert np.array_equal(from_bits.astype(np.float64), (2 * f.astype(np.float64) + 1) * 2.0 ** -22)


def test_direction_stream_layout():
    """The split walk's direction uniforms: Philox4x32-10 block k of domain 0
    (counter (k, 0, walker_lo, walker_hi), key = seed) serves steps 3k, 3k+1,
    3k+2 -- its 128 bits cut into six 21-bit fields from the top word down,
    fields 2j and 2j+1 for step 3k+j, field f read as (2f + 1) 2^-22."""
    seed, walker, nsteps = 0x1234ABCD5678EF01, 77, 31
    got = engine.rng_split(seed, walker, 0, 2 * nsteps)
    want = []
    for i in range(nsteps):
        b = [int(x) for x in pyoracle.philox4x32_10([i // 3, 0, walker & 0xFFFFFFFF, walker >> 32],
                                                   [seed & 0xFFFFFFFF, seed >> 32])]
        bits = (b[0] << 96) | (b[1] << 64) | (b[2] << 32) | b[3]
        f = [(bits >> (107 - 21 * m)) & 0x1FFFFF for m in range(6)]
        j = i % 3
        want += [(2 * f[2 * j] + 1) * 2.0 ** -22, (2 * f[2 * j + 1] + 1) * 2.0 ** -22]
    assert np.array_equal(got.astype(np.float64), np.array(want))
    assert np.array_equal(got, pyoracle.split_dir_uniforms(seed, walker, nsteps))
