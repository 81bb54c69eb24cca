"""GPU check of the row shards of the multi-GPU H-matvec, all shards in one
process: the shards' H*x add up to the full H*x (bit for bit: every row is
summed over the same leaves in the same order), their H'*x to the full H'*x,
and lu! refuses a shard."""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [2, 3])
def test_shards_add_up_to_the_full_matvec(world):
    import hmatrix as hm
    from hmatrix.shard import ShardedHmat
    n = 8192
    prm = hm.Params(Geom=np.linspace(0, 10, n), Kernel=hm.Cauchy(1.0), MaxBlock=512, MinBlock=64, MaxRank=16,
                    ConsMethod="aca2", εComp=1e-8, Tree="bisect")
    c, H = hm.NewHmat(dataclasses.replace(prm))
    shards = [ShardedHmat(dataclasses.replace(prm), r, world, cluster=c) for r in range(world)]
    assert shards[0].splits[0] == 0 and shards[-1].splits[-1] == n
    x = np.random.default_rng(3).standard_normal((n, 2))
    ys = [s.H * x for s in shards]
    assert np.array_equal(sum(ys), H * x)
    for s, y in zip(shards, ys):                 # each shard's rows, zeros elsewhere
        mask = np.ones(n, bool)
        mask[s.lo:s.hi] = False
        assert not y[mask].any()
    yt = sum(s.H.matvec(x, trans=True) for s in shards)
    assert np.linalg.norm(yt - H.matvec(x, trans=True)) <= 1e-13 * np.linalg.norm(yt)
    assert sum(s.H.info().n_rk for s in shards) == H.info().n_rk
    with pytest.raises(hm.HmError) as e:
        shards[0].H.lu_()
    assert "shard" in str(e.value)
