"""The breadth-first schedule of the split-radix tree and the level-pair
accounting of bench.py, on the CPU.

The library walks the reference's recursion (lab/parallel/mp/parallel_mp_fft2.c:
180-182: the n/2 child at out+0, the n/4 children at out+n/2 and out+3n/4)
and, for two levels run in one launch, pairs every node of size 2n with its
first child (the node of size n at the same offset) and runs the other nodes
of size n on their own.  These tests restate that walk and check the facts the
kernels and the bench's roofline rely on.
"""
import pytest


def _walk(n, out, levels, leaf_max=4):
    if n <= leaf_max:
        return
    _walk(n // 2, out, levels, leaf_max)
    _walk(n // 4, out + n // 2, levels, leaf_max)
    _walk(n // 4, out + 3 * n // 4, levels, leaf_max)
    levels.setdefault(n, []).append(out)


def _levels(N, leaf_max=4):
    levels = {}
    _walk(N, 0, levels, leaf_max)
    return dict(sorted(levels.items()))


@pytest.mark.parametrize("N", [8, 16, 64, 1024, 2048, 65536])
def test_first_children_start_at_parent_offsets(N):
    """Every node of size 2n has exactly one first child among the nodes of
    size n, at its own offset; the others are conjugate-pair children of
    nodes of size 4n."""
    lv = _levels(N)
    sizes = list(lv)
    for n, n2 in zip(sizes, sizes[1:]):
        assert n2 == 2 * n
        lower, upper = set(lv[n]), set(lv[n2])
        assert upper <= lower  # each parent offset is a child's offset
        others = lower - upper
        four = set(lv.get(4 * n, []))
        assert all(o - 2 * n in four or o - 3 * n in four for o in others)


@pytest.mark.parametrize("N", [16, 64, 1024, 2048, 65536])
def test_level_passes_touch_every_point_once(N):
    """bench.level_passes: with every other level folded into the one below
    it (a timed entry of 0), each launch touches all N points exactly once;
    with one level per launch a level touches count * n points."""
    import bench

    lv = _levels(N)
    sched = [(n, len(offs)) for n, offs in lv.items()]
    paired = [1.0 if i % 2 == 0 else 0.0 for i in range(len(sched))]  # pairs from the bottom
    passes = bench.level_passes(sched, paired)
    assert len(passes) == (len(sched) + 1) // 2
    assert all(pts == N for _, pts in passes)
    single = bench.level_passes(sched, [1.0] * len(sched))
    assert [pts for _, pts in single] == [n * c for n, c in sched]


def test_level_counts_match_the_op_count_known_answer():
    """The bench's product count per transform from the schedule: 7172 real
    multiplications at N=1024 (the reference's counter,
    lab/serial/mp/OPTIONS.md:42)."""
    import bench

    lv = _levels(1024)
    assert sum(len(offs) * bench.level_mults(n) for n, offs in lv.items()) == 7172
