"""Column-sharded K build over two CPU ranks (gloo): the host logic of the
multi-GPU path. Each rank's column solver here is the oracle's C restatement,
standing in for the GPU build; the gathered K must equal the single-process
build column for column (the reference's threaded-vs-serial K test,
test/fault_response_test.jl:100-112)."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, outdir):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    from datetime import timedelta
    from conftest import load_package
    from oracle.fault import FaultElasticity as OracleFE, cube_grids
    from oracle.cref import CRefStiffness

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        shard = sys.modules.get("eqd_b200.sharding")
        if shard is None:
            import importlib.util
            spec = importlib.util.spec_from_file_location(
                "eqd_sharding", os.path.join(ROOT, "earthquakediffinitive.jl_b200", "sharding.py"))
            shard = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(shard)
        gm, gp = cube_grids(11)
        ofe = OracleFE(gm, gp, 2.0, 1.0, l_f=0.4)
        ref = CRefStiffness(ofe)
        K, (lo, hi) = shard.fault_stiffness_sharded(ofe, build=lambda c: ref.columns(c, rtol=1e-12, nthreads=1)[0])
        t = shard.max_over_ranks(float(rank + 1))
        np.save(os.path.join(outdir, f"K{rank}.npy"), K)
        np.save(os.path.join(outdir, f"meta{rank}.npy"), np.array([lo, hi, t]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_build_gathers_full_K(tmp_path, world):
    import torch.multiprocessing as mp
    sys.path.insert(0, ROOT)
    from oracle.fault import FaultElasticity as OracleFE, cube_grids
    from oracle.cref import CRefStiffness

    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    gm, gp = cube_grids(11)
    ofe = OracleFE(gm, gp, 2.0, 1.0, l_f=0.4)
    K_ref = CRefStiffness(ofe).columns(np.arange(2 * ofe.nf), rtol=1e-12, nthreads=1)[0]
    covered = []
    for r in range(world):
        K = np.load(tmp_path / f"K{r}.npy")
        lo, hi, t = np.load(tmp_path / f"meta{r}.npy")
        assert np.array_equal(K, K_ref)          # every rank holds the full K
        assert t == world                         # max over ranks
        covered += list(range(int(lo), int(hi)))
    assert covered == list(range(2 * ofe.nf))    # contiguous, disjoint, complete


def test_shard_range_edges():
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "eqd_sharding", os.path.join(ROOT, "earthquakediffinitive.jl_b200", "sharding.py"))
    shard = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(shard)
    for n in (0, 1, 7, 50, 2178):
        for w in (1, 2, 3, 8):
            blocks = [shard.shard_range(n, r, w) for r in range(w)]
            assert blocks[0][0] == 0 and blocks[-1][1] == n
            assert all(blocks[i][1] == blocks[i + 1][0] for i in range(w - 1))
            assert max(b - a for a, b in blocks) - min(b - a for a, b in blocks) <= 1
    with pytest.raises(ValueError):
        shard.shard_range(10, 2, 2)
