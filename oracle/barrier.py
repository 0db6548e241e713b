"""Serial host restatement of the remapping-barrier workload — TEST INFRASTRUCTURE ONLY.

Follows harmonize examples/cpp/barrier_demo/demo.cpp:20-86 and :163-170 (one Step per id in
[0, dep + ndep); a dependent id holds a follow-up Step on barrier id % bar and then
decrements it; barrier b starts at the number of dependent ids congruent to b) and
sync/barrier.h:460-639 (held promises run once the semaphore reaches zero), with the
additions of the GPU workload (harmonize_b200/csrc/specs/barrier_demo.h): follow-ups count
themselves per barrier, and a unit barrier armed with ndep releases one final Step.
Pure Python: for small cases.
"""
from collections import deque

FOLLOW = 0x80000000
FINAL = 0x7FFFFFFF


def barrier_demo(dep, ndep, bar):
    """Returns (counter[4], released[bar]) exactly as the GPU run must report them."""
    sem = [dep // bar + (1 if (dep % bar) > b else 0) for b in range(bar)]
    held = [[] for _ in range(bar)]
    unit = ndep
    counter = [0, 0, 0, 0]
    released = [0] * bar
    queue = deque(range(dep + ndep))
    while queue:
        arg = queue.popleft()
        counter[0] += 1
        if arg >= FOLLOW:
            b = arg - FOLLOW
            released[b] += 1
            if sem[b] != 0:
                counter[3] += 1
        elif arg == FINAL:
            counter[2] += 1
            if counter[1] != ndep:
                counter[3] += 1
        elif arg < dep:
            b = arg % bar
            if sem[b] == 0:
                queue.append(FOLLOW + b)
            else:
                held[b].append(FOLLOW + b)
            sem[b] -= 1
            if sem[b] == 0:
                queue.extend(held[b])
                held[b] = []
        else:
            counter[1] += 1
            unit -= 1
            if unit == 0:
                queue.append(FINAL)
    return counter, released
