"""The device planted-partition batch generator (gpu_build.sbm_batch) draws
each instance's size, block count and degrees exactly as the host generator
graphs.sbm_batch does (same per-instance random stream), so the two batches
have the same instances and vertex ranges; only the edge samples differ."""
import numpy as np

from parex_b200 import gpu_build as B
from parex_b200 import graphs as G


def test_device_batch_parameters_match_the_host_generator():
    g, starts = G.sbm_batch(count=6, seed=4, n_lo=50, n_hi=400)
    params = B.sbm_batch_params(count=6, seed=4, n_lo=50, n_hi=400)
    sizes = np.array([p[0] for p in params], dtype=np.int64)
    np.testing.assert_array_equal(np.diff(starts), sizes)
    assert g.n == int(sizes.sum())
    for n, blocks, d_in, d_out in params:
        assert 2 <= blocks <= 64 and blocks <= max(1, n // 2)
        assert 4.0 <= d_in <= 32.0 and 0.1 <= d_out <= 2.0


def test_sampler_work_list_covers_every_vertex_pair_once():
    params = B.sbm_batch_params(count=5, seed=2, n_lo=30, n_hi=300)
    T, prefix, starts = B.sbm_batch_tasks(params, segment_len=64)
    su = T["su"].astype(np.int64)
    sv = T["sv"].astype(np.int64)
    cand = np.where(T["intra"] == 1, su * (su - 1) // 2, su * sv)
    # the block pairs of an instance cover its n (n - 1) / 2 vertex pairs exactly
    inst = np.searchsorted(np.asarray(starts), T["base_u"].astype(np.int64), side="right") - 1
    for i, (n, blocks, _, _) in enumerate(params):
        assert int(cand[inst == i].sum()) == n * (n - 1) // 2
        assert int(np.count_nonzero(inst == i)) == blocks * (blocks + 1) // 2
    # both blocks of a task lie inside the task's instance
    end = np.asarray(starts)[inst + 1]
    assert np.all(T["base_u"].astype(np.int64) + su <= end) and np.all(T["base_v"].astype(np.int64) + sv <= end)
    # segments: non-decreasing first segments, enough segments for every task's pairs
    nseg = np.diff(prefix.astype(np.int64))
    assert np.all(nseg >= 0) and np.all(nseg * 64 >= cand) and np.all((nseg - 1) * 64 < np.maximum(cand, 1))
    assert np.all(T["p"] > 0) and np.all(T["p"] <= 1)


def test_shards_partition_the_batch_and_balance_expected_edges():
    params = B.sbm_batch_params(count=512, seed=1)
    weight = np.array([n * (a + b) / 2 for n, _, a, b in params])
    for world in (1, 2, 4, 8):
        shards = B.shard_instances(params, world)
        assert len(shards) == world
        allidx = np.sort(np.concatenate([np.asarray(s, dtype=np.int64) for s in shards]))
        np.testing.assert_array_equal(allidx, np.arange(512))
        loads = np.array([weight[s].sum() for s in shards])
        assert loads.max() - loads.min() <= weight.max() + 1e-6   # greedy bound
        assert shards == B.shard_instances(params, world)          # deterministic


def test_a_shard_holds_the_same_tasks_as_the_whole_batch():
    params = B.sbm_batch_params(count=6, seed=4, n_lo=40, n_hi=400)
    T, _, starts = B.sbm_batch_tasks(params, 64)
    Ts, _, starts_s = B.sbm_batch_tasks(params, 64, instances=[1, 4])
    full_inst = np.searchsorted(np.asarray(starts), T["base_u"].astype(np.int64), side="right") - 1
    sub = T[np.isin(full_inst, [1, 4])]
    for f in ("su", "sv", "p", "intra", "key"):
        np.testing.assert_array_equal(Ts[f], sub[f])
    # vertex bases move with the instance's place in the shard
    n1 = params[1][0]
    off = np.where(np.arange(len(sub)) < np.count_nonzero(full_inst == 1), starts[1], starts[4] - n1)
    np.testing.assert_array_equal(Ts["base_u"].astype(np.int64), sub["base_u"].astype(np.int64) - off)
    assert starts_s == [0, n1, n1 + params[4][0]]
