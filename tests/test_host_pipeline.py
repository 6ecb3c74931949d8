"""Chunking of the host-memory pipeline (eval_host): the chunks tile [0, N) in order,
never exceed the buffer size, and ramp up and down around full-size chunks."""
import pytest

from agama_gpu_b200.potentials import _chunk_bounds


@pytest.mark.parametrize("n,chunk", [(4_000_000, 1 << 20), (100_003, 30_000), (100_003, 1 << 19),
                                     (2_500_000, 1 << 20), (2 * (1 << 20) + 1, 1 << 20), (5, 2),
                                     (1, 1), (0, 7), (3 * 4096 + 17, 4096)])
def test_chunks_tile_the_range(n, chunk):
    b = _chunk_bounds(n, chunk)
    assert sum(h - l for l, h in b) == n
    assert all(h > l for l, h in b)
    assert all(b[i][1] == b[i + 1][0] for i in range(len(b) - 1))
    assert not b or (b[0][0] == 0 and b[-1][1] == n)
    assert all(h - l <= chunk for l, h in b)


def test_ramp_shape():
    sizes = [h - l for l, h in _chunk_bounds(4_000_000, 1 << 20)]
    assert sizes[:2] == [1 << 18, 1 << 19] and sizes[-3:] == [1 << 19, 1 << 18, 1 << 17]
    assert max(sizes) - min(sizes[2:-3]) <= 1            # the full-size middle is evened out


WAVE = 148 * 2 * 256          # a B200 wave of the Phi+F kernel (2 resident blocks per SM)


@pytest.mark.parametrize("n,chunk,wave", [(4_000_000, 1 << 20, WAVE), (4_194_304, 1 << 20, WAVE),
                                          (40_000_003, 1 << 20, WAVE), (1_000_000, 333_334, WAVE),
                                          (3_000_000, 1_000_000, WAVE), (700_001, 1 << 17, 4096),
                                          (100_003, 30_000, 60_000), (5, 2, 1), (0, 7, 3)])
def test_wave_chunks_tile_the_range(n, chunk, wave):
    b = _chunk_bounds(n, chunk, wave)
    assert sum(h - l for l, h in b) == n
    assert all(h > l for l, h in b)
    assert all(b[i][1] == b[i + 1][0] for i in range(len(b) - 1))
    assert not b or (b[0][0] == 0 and b[-1][1] == n)
    sizes = [h - l for l, h in b]
    if n >= 20 * wave and chunk >= wave:
        # every chunk but the last is whole waves, the last holds 2 to 3 waves
        assert all(m % wave == 0 for m in sizes[:-1])
        assert 2 * wave <= sizes[-1] < 3 * wave
        assert max(sizes) <= round(chunk / wave) * wave


def test_wave_ramp_shape():
    sizes = [(h - l) / WAVE for l, h in _chunk_bounds(4_000_000, 1 << 20, WAVE)]
    assert sizes[:-1] == [2, 6, 14, 14, 10, 4]
    assert 2 <= sizes[-1] < 3
