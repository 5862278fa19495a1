"""BitVoxelMap bit maintenance in the oracle: performLeftShift pinned by the
known answers of the reference's test (GV/test/testing_bitvector.cu,
bitvector_bitshift), and its byte-buffer loop shown equal to a plain 256-bit
right shift with meanings 0..3 cleared (the form the GPU kernel computes)."""
import numpy as np
import pytest

import oracle


def _vec(bits):
    v = np.zeros(32, dtype=np.uint8)
    for b in bits:
        v[b >> 3] |= np.uint8(1 << (b & 7))
    return v


def _bits(v):
    return {b for b in range(256) if v[b >> 3] >> (b & 7) & 1}


@pytest.mark.parametrize("shift", [3, 13])
def test_reference_known_answers(shift):
    v = _vec([0, 1, 2, 3, 4, 14, 24, 254, 255])
    oracle.bvm_shift(v, shift)
    got = _bits(v)
    assert not got & {0, 1, 2, 3, 4, 14, 24, 254, 255}
    assert (24 - shift in got) == (24 - shift > 3)
    assert 254 - shift in got and 255 - shift in got


def test_byte_loop_is_a_256_bit_shift():
    rng = np.random.default_rng(0)
    maps = rng.integers(0, 256, size=(64, 32)).astype(np.uint8)
    for shift in list(range(0, 57)):
        m = maps.copy().reshape(-1)
        oracle.bvm_shift(m, shift)
        for k in range(64):
            x = int.from_bytes(maps[k].tobytes(), "little")
            want = ((x >> shift) & ~0xF).to_bytes(32, "little")
            assert m[32 * k:32 * k + 32].tobytes() == want, (shift, k)


def test_clear_bits():
    m = np.stack([_vec([1, 5, 200]), _vec([7]), _vec([])]).reshape(-1)
    oracle.bvm_clear_bits(m, _vec([5, 7, 9]))
    v = m.reshape(3, 32)
    assert _bits(v[0]) == {1, 200} and _bits(v[1]) == set() and _bits(v[2]) == set()
