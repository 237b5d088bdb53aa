"""Batched design jobs: every instance's result in the batch equals the same job run alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

JOBS = [  # L (aa, without stop), m, N, objective set, seed
    (150, 2, 64, 1, 11),
    (400, 4, 128, 1, 12),
    (90, 8, 32, 0, 13),
    (700, 3, 96, 1, 14),
]


def make(pe, ref_table, L, m, N, objset, seed):
    tab = ref_table if objset == 0 else pe.dirichlet_table(seed)
    eng = pe.Engine(pe.synthetic_protein(L, seed), tab, m, N, 0.03, objectives=objset, seed=seed)
    eng.init()
    return eng


def test_batch_equals_alone(pe, ref_table, gpu):
    alone = []
    for job in JOBS:
        with make(pe, ref_table, *job) as e:
            e.step(7)
            alone.append(e.population())
    engines = [make(pe, ref_table, *job) for job in JOBS]
    with pe.Batch(engines) as b:
        b.step(3)       # 2 + 1 generations
        b.step(4)       # parity changed: graphs rebuilt
        b.synchronize()
    for e, want in zip(engines, alone):
        got = e.population()
        assert e.generation == 7
        for k in range(5):
            a, w = np.asarray(got[k]), np.asarray(want[k])
            if a.dtype.kind == "f":
                a, w = a.view(np.uint32), w.view(np.uint32)
            assert np.array_equal(a, w)
        e.close()


def test_batch_then_single_steps_stay_ordered(pe, ref_table, gpu):
    e1 = make(pe, ref_table, 120, 2, 32, 1, 5)
    e2 = make(pe, ref_table, 120, 2, 32, 1, 5)
    with pe.Batch([e1]) as b:
        b.step(2)
    e1.step(1)                      # on the member's own stream, after the batch
    e2.step(3)
    for k in range(5):
        assert np.array_equal(np.asarray(e1.population()[k]), np.asarray(e2.population()[k]))
    e1.close()
    e2.close()
