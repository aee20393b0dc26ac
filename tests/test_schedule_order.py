"""The dependency rules of the persistent relaxation kernel preserve the reference order.

The kernel runs task (slice z, visit t) once visit t of z+1, visit t-1 of z-1 and visit t-1
of z are done.  Any execution honouring those edges must give every coupled slice pair
(z, z+1) the visit sequence of the sequential order (warp-psr relaxation.py:121-143,
tests/test_relaxation.py:94-107).  Random valid executions are simulated on the CPU.
"""
import random

import pytest


def sequential(depth, iters):
    n = 1 << depth
    out = []
    for front in range(n, -iters, -1):
        for z in range(max(front, 0), min(front + iters, n + 1)):
            out.append((z, z - front))
    return out


def random_execution(depth, iters, rng):
    n = 1 << depth
    done = {z: 0 for z in range(n + 1)}  # visits completed per slice
    pending = sequential(depth, iters)
    order = []
    while pending:
        ready = [(z, t) for (z, t) in pending
                 if done[z] == t and (z + 1 > n or done[z + 1] >= t + 1) and (z == 0 or done[z - 1] >= t)]
        assert ready, "dependency rules deadlocked"
        task = rng.choice(ready)
        pending.remove(task)
        done[task[0]] += 1
        order.append(task)
    return order


@pytest.mark.parametrize("depth", [0, 1, 3, 4])
@pytest.mark.parametrize("iters", [1, 3, 8])
def test_every_coupled_pair_keeps_its_visit_sequence(depth, iters):
    rng = random.Random(depth * 100 + iters)
    seq = sequential(depth, iters)
    for _ in range(5):
        par = random_execution(depth, iters, rng)
        assert sorted(par) == sorted(seq)
        for z in range(1 << depth):
            pair = (z, z + 1)
            assert [t for t in par if t[0] in pair] == [t for t in seq if t[0] in pair]


def wave_order(depth, iters):
    n = 1 << depth
    out = []
    for q in range(n + 2 * (iters - 1) + 1):
        first, last = max(0, (q - n + 1) // 2), min(iters - 1, q // 2)
        out.extend((n - q + 2 * t, t) for t in range(first, last + 1))
    return out


@pytest.mark.parametrize("depth", [0, 1, 3, 5, 9])
@pytest.mark.parametrize("iters", [1, 2, 8])
def test_wave_dequeue_order_is_complete_and_deadlock_free(depth, iters):
    seq = sequential(depth, iters)
    waves = wave_order(depth, iters)
    assert sorted(waves) == sorted(seq) and len(set(waves)) == len(waves)
    pos = {task: i for i, task in enumerate(waves)}
    for (z, t), i in pos.items():
        for dep in ((z + 1, t), (z - 1, t - 1), (z, t - 1)):
            if dep in pos:
                assert pos[dep] < i


def test_tasks_only_wait_on_earlier_tasks():
    # Deadlock freedom: every dependency of a task precedes it in the dequeue order.
    for depth in range(6):
        for iters in (1, 2, 8):
            seq = sequential(depth, iters)
            pos = {task: i for i, task in enumerate(seq)}
            n = 1 << depth
            for (z, t), i in pos.items():
                for dep in ((z + 1, t), (z - 1, t - 1), (z, t - 1)):
                    if dep in pos:
                        assert pos[dep] < i
