"""Multi-rank orientation sharding (one process per GPU in production),
exercised as world_size-2 gloo ranks on the CPU with the oracle standing in
for the device call.  Also the host-side failure paths: a rank whose call
fails, and a rank that dies before the reduction."""
import os
import socket

import numpy as np
import pytest

from mbs_fast_b200 import shard


def test_orientation_range_partitions_like_the_reference():
    for n in (0, 1, 7, 16384):
        for world in (1, 2, 3, 8):
            got = [shard.orientation_range(n, r, world, start=5) for r in range(world)]
            assert got[0][0] == 5
            for (b0, c0), (b1, _) in zip(got, got[1:]):
                assert b0 + c0 == b1
            assert sum(c for _, c in got) == n
            assert max(c for _, c in got) - min(c for _, c in got) <= 1
    with pytest.raises(ValueError):
        shard.orientation_range(4, 2, 2)


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


class _OracleHandler:
    """Stand-in for GpuHandlerPO on a CPU rank: the oracle does the work."""

    def __init__(self, grid, wave, fail=False):
        self.grid, self.wave, self.fail = grid, wave, fail

    def handle_orientations_to_local_gpu(self, batch, m, mns=None, start=0, count=None,
                                         precision=0):
        import oracle
        if self.fail:
            return False
        part = batch.select(start, count)
        out = oracle.po_diffract(part, self.grid, self.wave, n_threads=1, noshadow=mns is not None)
        if mns is not None:
            m += out[0]
            mns += out[1]
        else:
            m += out
        return True


def _rank_main(rank, world, port, outdir, mode):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=20))
    from mbs_fast_b200 import beams as B
    from tests import common
    batch = common.sobol_batch("hex10x20", 5)
    grid = B.grid(0.0, 180.0, 6, 40)
    wave = B.wave(common.HEX_COLUMN_10x20)
    if mode == "dead" and rank == 1:
        os._exit(0)           # leaves between steps, before the reduction
    h = _OracleHandler(grid, wave, fail=(mode == "fail" and rank == 1))
    m = np.zeros((grid.n_az, grid.n_zen + 1, 16))
    mns = np.zeros_like(m)
    try:
        ok = shard.diffract_sharded(h, batch, m, mns, rank=rank, world=world)
        np.save(os.path.join(outdir, f"m{rank}.npy"), m)
        np.save(os.path.join(outdir, f"mns{rank}.npy"), mns)
        with open(os.path.join(outdir, f"ok{rank}"), "w") as f:
            f.write("1" if ok else "0")
    except Exception as e:   # a dead peer surfaces as an error, not a hang
        with open(os.path.join(outdir, f"err{rank}"), "w") as f:
            f.write(type(e).__name__ + ": " + str(e)[:200])
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _spawn(mode, tmp_path):
    import torch.multiprocessing as mp
    import time
    ctx = mp.spawn(_rank_main, args=(2, _free_port(), str(tmp_path), mode), nprocs=2,
                   join=False)
    deadline = time.time() + 120
    # join() returns after any one process ends; wait for all of them
    while not ctx.join(timeout=5) and time.time() < deadline:
        pass
    for p in ctx.processes:
        if p.is_alive():
            p.kill()
    return tmp_path


def test_sharded_sum_equals_whole_batch(tmp_path):
    import oracle
    from mbs_fast_b200 import beams as B
    from tests import common
    _spawn("ok", tmp_path)
    batch = common.sobol_batch("hex10x20", 5)
    grid = B.grid(0.0, 180.0, 6, 40)
    want, want_ns = oracle.po_diffract(batch, grid, B.wave(common.HEX_COLUMN_10x20),
                                       noshadow=True)
    for r in range(2):
        assert (tmp_path / f"ok{r}").read_text() == "1"
        m = np.load(tmp_path / f"m{r}.npy")
        mns = np.load(tmp_path / f"mns{r}.npy")
        assert np.max(np.abs(m - want)) <= 1e-12 * np.max(np.abs(want))
        assert np.max(np.abs(mns - want_ns)) <= 1e-12 * np.max(np.abs(want_ns))


def test_failed_rank_is_agreed_by_all(tmp_path):
    _spawn("fail", tmp_path)
    for r in range(2):
        assert (tmp_path / f"ok{r}").read_text() == "0"
        assert not np.load(tmp_path / f"m{r}.npy").any()   # nothing added on failure


def test_dead_rank_surfaces_as_error(tmp_path):
    _spawn("dead", tmp_path)
    assert (tmp_path / "err0").exists()
    assert not (tmp_path / "ok0").exists()
