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


def population_equal(got, want):
    for k in range(5):
        a, w = np.asarray(got[k]), np.asarray(want[k])
        if a.dtype.kind == "f":
            a, w = a.view(np.uint32), w.view(np.uint32)
        if not np.array_equal(a, w):
            return False
    return True


@pytest.mark.parametrize("queue", [True, False])
def test_queued_scan_classes_equal_alone(pe, ref_table, gpu, queue):
    """Members of three scan classes (forced CTA sizes 64, 128, 256) and both string
    objectives, with the batch's queued scan on and off: each equals its job alone."""
    jobs = [  # L, m, N, objective set, seed, scan CTA size, string objective
        (300, 3, 64, 1, 21, 64, pe.SL_HAIRPIN),
        (900, 2, 48, 1, 22, 256, pe.SL_HAIRPIN),
        (120, 4, 32, 0, 23, 128, pe.SL_HAIRPIN),
        (200, 3, 32, 1, 24, 128, pe.SL_LRCS),
        (60, 2, 32, 1, 25, 64, pe.SL_HAIRPIN),
    ]

    def mk(L, m, N, objset, seed, nt, kind):
        tab = ref_table if objset == 0 else pe.dirichlet_table(seed)
        e = pe.Engine(pe.synthetic_protein(L, seed), tab, m, N, 0.04, objectives=objset, seed=seed, sl_threads=nt,
                      sl_kind=kind)
        e.init()
        return e

    alone = []
    for job in jobs:
        with mk(*job) as e:
            e.step(6)
            alone.append(e.population())
    engines = [mk(*job) for job in jobs]
    with pe.Batch(engines) as b:
        b.set_scan_queue(queue)
        b.step(2)
        b.step(1)
        b.set_scan_queue(not queue)    # switching rebuilds the graphs; results do not change
        b.step(3)
        b.synchronize()
    for q, (e, want) in enumerate(zip(engines, alone)):
        assert e.generation == 6
        got = e.population()
        for k, what in enumerate(("codons", "obj", "objidx", "pql", "survivors")):
            assert population_equal([got[k]] * 5, [want[k]] * 5), f"member {q}: {what} differ"
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
