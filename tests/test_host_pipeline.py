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
