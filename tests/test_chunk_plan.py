"""Chunk plan of the streamed host path (runtime._chunk_bounds), which splits
the rays of one solve() call into consecutive chunks: the bounds start at 0,
end at n and never decrease; no chunk holds more than the chunk size asked
for; when the rays exceed eight end chunks, the first and the last chunk hold
STREAM_END_RAYS (the copies no trace hides); the other chunks are within one
ray of each other."""
from hypothesis import given, settings, strategies as st

from sloth_b200 import runtime

END = runtime.STREAM_END_RAYS


def _check(n, cs):
    b = runtime._chunk_bounds(n, cs)
    assert b[0] == 0 and b[-1] == max(n, 0)
    sizes = [hi - lo for lo, hi in zip(b, b[1:])]
    assert all(s >= 0 for s in sizes)
    assert max(sizes) <= max(cs, 0) or n <= 0
    if n > 0:
        assert all(s > 0 for s in sizes), (n, cs, sizes)
    end = min(cs, END)
    mid = sizes
    if n > 8 * end:
        assert sizes[0] == end and sizes[-1] == end
        mid = sizes[1:-1]
    if n > 0:
        assert max(mid) - min(mid) <= 1
        assert len(mid) == -(-sum(mid) // cs)
    return sizes


@st.composite
def _plans(draw):
    """A chunk size and a ray count of at most 64 middle chunks."""
    cs = draw(st.integers(min_value=1, max_value=1 << 24))
    n = draw(st.integers(min_value=0, max_value=64 * cs + 2 * min(cs, END)))
    return n, cs


@settings(max_examples=400, deadline=None)
@given(_plans())
def test_chunk_bounds_properties(plan):
    _check(*plan)


def test_chunk_bounds_bench_workload():
    """1e7 rays at the default chunk size: 0.5M, 9.0M, 0.5M."""
    sizes = _check(10_000_000, runtime.STREAM_CHUNK_RAYS)
    assert sizes[0] == sizes[-1] == END == 1 << 19
    assert len(sizes) == 3 and sum(sizes) == 10_000_000


def test_chunk_bounds_small_and_empty():
    assert runtime._chunk_bounds(0, 1 << 22) == [0, 0]
    assert _check(1, 1 << 22) == [1]
    assert _check(1 << 22, 1 << 22) == [1 << 22]
    assert _check(8 * END, 1 << 22) == [1 << 22]
    assert _check(8 * END + 1, 1 << 22) == [END, 6 * END + 1, END]
    assert _check(8 * END + 1, 1 << 21) == [END, 3 * END + 1, 3 * END, END]
