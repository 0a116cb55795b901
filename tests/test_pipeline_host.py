"""Host logic of the tracing pipeline (CPU): the batch boundaries cover the
orientations exactly once, in order, with a short first and last batch."""
import pytest

from mbs_fast_b200.pipeline import batch_edges


@pytest.mark.parametrize("n,batch", [(16384, 1024), (2048, 1024), (1000, 1024), (5000, 1024),
                                     (1536, 1024), (1, 8), (0, 8), (17, 4)])
def test_batch_edges_partition(n, batch):
    e = batch_edges(n, batch)
    assert e[0] == 0 and e[-1] == n
    sizes = [b - a for a, b in zip(e[:-1], e[1:])]
    assert all(s > 0 for s in sizes) and sum(sizes) == n
    assert all(s <= batch for s in sizes)
    if n > batch:
        assert sizes[0] <= batch // 4 + 1 and sizes[-1] <= batch // 2
