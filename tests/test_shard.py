"""Multi-GPU sharding of the batched form (pywignercuda_b200/shard.py), on the
CPU: the cost-balanced partition of the instances, and -- as two gloo ranks --
the gather of the per-instance observables to rank 0 and the bench's
max-over-ranks timing reduction."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from pywignercuda_b200.shard import gather_observables, imbalance, instance_cost, partition


def _batch():
    import bench
    return [dict(n_x=c['n'], n_p=c['n'], gamma=c['gamma']) for c in bench.batch_config()]


@pytest.mark.parametrize('world', [1, 2, 4, 8])
def test_partition_covers_every_instance_once(world):
    inst = _batch()
    parts = partition(inst, world)
    assert len(parts) == world
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(inst)))
    assert all(p == sorted(p) for p in parts)
    # LPT: the heaviest rank exceeds the mean by at most one instance's cost
    loads = [sum(instance_cost(inst[i]) for i in p) for p in parts]
    assert max(loads) - np.mean(loads) <= max(instance_cost(d) for d in inst) + 1e-6
    if world <= 4:
        assert imbalance(inst, parts) < 1.10


def test_cost_uses_the_measured_table():
    from pywignercuda_b200.shard import MEASURED_NS
    for d in _batch():
        key = '%d%s' % (d['n_x'], 'd' if d['gamma'] else '')
        assert key in MEASURED_NS
        assert instance_cost(d) == pytest.approx(d['n_x'] * d['n_p'] * MEASURED_NS[key])
    # a size class outside the table: the transform-count model, damped four times the undamped
    und, dmp = dict(n_x=2048, n_p=64, gamma=0.), dict(n_x=2048, n_p=64, gamma=0.1)
    assert instance_cost(dmp) == pytest.approx(4. * instance_cost(und))
    # a caller's own table takes precedence
    assert instance_cost(dict(n_x=128, n_p=128, gamma=0.), {'128': 2.}) == pytest.approx(2. * 128 * 128)


def test_partition_is_deterministic():
    inst = _batch()
    assert partition(inst, 4) == partition(inst, 4)


def _obs_of(i, n=6):
    return np.full((n, 11), float(i)) + np.arange(11)[None, :] * 1e-3


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    import bench
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        inst = _batch()
        parts = partition(inst, world)
        local = np.stack([_obs_of(i) for i in parts[rank]])
        full = gather_observables(local, parts, rank)
        if rank == 0:
            assert full.shape == (len(inst), 6, 11)
            for i in range(len(inst)):
                assert np.array_equal(full[i], _obs_of(i)), i
        else:
            assert full is None
        ms = bench.barrier_max(world, 10. + rank)
        assert ms == 10. + (world - 1)
        bench.barrier(world)
        open(os.path.join(out_dir, 'ok%d' % rank), 'w').write('ok')
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def test_gloo_two_ranks_gather_and_max(tmp_path):
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    assert sorted(os.listdir(tmp_path)) == ['ok0', 'ok1']


def _val(rank):
    leg = lambda e: {'steps': 2000, 'norm_max_abs': 1e-16 * (rank + 1), 'energy_rel_max': e,
                     'energy_rel_final': 2 * e, 'state_rel_l2_final': 3 * e}
    dw = {'steps': 4000, 'norm_max_abs': 1e-16, 'energy_rel_max': 4e-9, 'energy_rel_final': 1e-9,
          'state_rel_l2_final': 1e-7}
    return {'mixed': {'batch_2000': leg(1e-7 * (rank + 1)), 'double_well_1024_4000': dict(dw)},
            'f32': {'batch_2000': leg(1e-3 / (rank + 1)), 'double_well_1024_4000': dict(dw)},
            'reference': 'text'}


def _merge_main(rank, world, port, out_dir):
    import json
    import torch.distributed as dist
    import bench
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        merged = bench.merge_validation(_val(rank), world)
        open(os.path.join(out_dir, 'm%d.json' % rank), 'w').write(json.dumps(merged))
    finally:
        dist.destroy_process_group()


def test_gloo_validation_merged_on_every_rank(tmp_path):
    """bench.merge_validation: each rank validates its own share of the batch; every
    rank gets the worst batch figures over the ranks (so all ranks pick the same
    headline form) and the double-well leg as run."""
    import json
    world = 2
    mp.spawn(_merge_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    m0, m1 = (json.loads(open(os.path.join(tmp_path, 'm%d.json' % r)).read()) for r in range(world))
    assert m0 == m1
    assert m0['mixed']['batch_2000']['energy_rel_max'] == pytest.approx(2e-7)
    assert m0['f32']['batch_2000']['energy_rel_max'] == pytest.approx(1e-3)
    assert m0['mixed']['batch_2000']['steps'] == 2000
    assert m0['mixed']['double_well_1024_4000']['energy_rel_max'] == pytest.approx(4e-9)
    assert m0['reference'] == 'text'
    assert bench_merge_single() is None


def bench_merge_single():
    import bench
    assert bench.merge_validation({'a': 1}, 1) == {'a': 1}
    return bench.merge_validation(None, 2)
