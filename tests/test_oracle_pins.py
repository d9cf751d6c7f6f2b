"""Pins the oracle (the reference compiled from its own sources) before it is
trusted: its RNG and hash against the published PCG32 / MurmurHash64A
definitions restated here, the workload generator's PCG32 streams, and the
README scene against the value the reference produced when first built here
(mean luminance 0.131778 at 320x180, 16 spp, 8 bounces)."""
import numpy as np

from bulbit_b200 import scenes

M64 = (1 << 64) - 1


def pcg32_py(initstate, initseq, n):
    """PCG32 (pcg-random.org, pcg32_srandom_r / pcg32_random_r)."""
    mult = 0x5851F42D4C957F2D
    inc = ((initseq << 1) | 1) & M64
    state = 0

    def step(st):
        old = st
        st = (old * mult + inc) & M64
        xs = (((old >> 18) ^ old) >> 27) & 0xFFFFFFFF
        rot = old >> 59
        return st, ((xs >> rot) | (xs << ((-rot) & 31))) & 0xFFFFFFFF

    state, _ = step(state)
    state = (state + initstate) & M64
    state, _ = step(state)
    out = []
    for _ in range(n):
        state, v = step(state)
        out.append(v)
    return out


def murmur64a_py(data, seed=0):
    """MurmurHash64A (Austin Appleby), little-endian, for len % 8 == 0."""
    m, r = 0xC6A4A7935BD1E995, 47
    h = (seed ^ (len(data) * m)) & M64
    for i in range(0, len(data), 8):
        k = int.from_bytes(data[i:i + 8], "little")
        k = (k * m) & M64
        k ^= k >> r
        k = (k * m) & M64
        h ^= k
        h = (h * m) & M64
    h ^= h >> r
    h = (h * m) & M64
    h ^= h >> r
    return h


def test_oracle_pcg32_matches_published_definition(oracle):
    for state, seq in [(0, 1), (42, 54), (0xDEADBEEF, 1), (2**63 + 7, 12345)]:
        assert oracle.pcg32(state, seq, 16).tolist() == pcg32_py(state, seq, 16)


def test_pcg32_known_answer(oracle):
    # pcg32-demo reference output for pcg32_srandom(42, 54).
    assert oracle.pcg32(42, 54, 6).tolist() == [0xA15C02B7, 0x7B47F409, 0xBA1D3330, 0x83D2F293,
                                                0xBFA4784B, 0xCBED606E]


def test_oracle_pixel_hash_matches_murmur(oracle):
    import struct
    for px, py, seed, s in [(0, 0, 0, 0), (319, 179, 0, 15), (12, 7, 5, 3), (1023, 1023, 0, 63)]:
        data = struct.pack("<iiii", px, py, seed, s)
        assert oracle.hash_pixel_sample(px, py, seed, s) == murmur64a_py(data)


def test_oracle_sampler_draws_are_pcg32_of_pixel_hash(oracle):
    import struct
    px, py, seed, s = 5, 9, 0, 2
    h = murmur64a_py(struct.pack("<iiii", px, py, seed, s))
    u = np.array(pcg32_py(h, 1, 8), np.uint32).astype(np.float32) * np.float32(2.0 ** -32)
    u = np.minimum(np.float32(1) - np.finfo(np.float32).eps, u)
    assert np.array_equal(oracle.sampler_draws(px, py, seed, s, 8), u)


def test_generator_streams_are_reference_pcg32(oracle):
    g = scenes.PCG32Streams(7, np.arange(5, dtype=np.uint64))
    vals = np.stack([g.next_uint() for _ in range(4)], axis=1)
    for i in range(5):
        assert vals[i].tolist() == oracle.pcg32(7, i, 4).tolist()


def test_readme_scene_luminance_pinned(oracle):
    rs = oracle.RefScene(scenes.readme_sphere())
    rs.make_integrator()
    img, _, _ = rs.render()
    lum = 0.2126 * img[..., 0] + 0.7152 * img[..., 1] + 0.0722 * img[..., 2]
    assert abs(float(lum.mean()) - 0.131778) < 5e-7
