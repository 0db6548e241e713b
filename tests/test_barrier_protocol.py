"""A model of RemappingBarrier's held-link protocol (include/harmonize/barrier.h), run under many
random interleavings on the CPU: every promise awaited on the barrier must come out exactly
once, either passed straight on (the barrier had already released) or published in a held
link after the release, whatever the order in which warps reserve, write, retire links,
release and sweep, while published links are consumed and returned to the free pool. A
release may come while groups are between their reservation and their writes: the sweep then
waits for the writes, and a group that finishes after the release sweeps for itself.

Each actor is a generator that yields between its shared-memory steps (the atomic
operations and stores of the CUDA code); a seeded scheduler picks which actor steps next.
Leaving out the wait for writers, the retirement of replaced links or the awaiter's own
sweep makes hundreds of the seeds fail.
"""
import random

SLOTS = 32


class World:
    def __init__(self, n_links, sem):
        self.partial = (0, 0, 0)           # (tag, reserved, link + 1)
        self.head = 0                      # retired stack: link + 1
        self.next = {}                     # link -> (next link + 1, reserved)
        self.written = {}                  # link -> promises written
        self.slots = {}                    # link -> {slot: promise}
        self.free = list(range(n_links))
        self.sem = sem
        self.out = []                      # promises that came out (direct or published)
        self.queue = []                    # published links not yet consumed

    def cas_partial(self, old, new):
        if self.partial == old:
            self.partial = new
            return True
        return False


def publish_held(w, link, reserved):
    while w.written[link] < reserved:      # bounded in the CUDA code; here the writers always finish
        yield
    w.out.extend(w.slots[link][s] for s in range(reserved))
    w.queue.append(link)


def sweep(w):
    # the partial link
    while True:
        old = w.partial
        yield
        if old[2] == 0:
            break
        if w.cas_partial(old, (old[0] + 1, 0, 0)):
            yield from publish_held(w, old[2] - 1, old[1])
            break
    # the retired stack
    h, w.head = w.head, 0
    yield
    while h:
        link = h - 1
        nxt, reserved = w.next[link]
        yield from publish_held(w, link, reserved)
        h = nxt


def retire(w, link, reserved):
    while True:
        old = w.head
        w.next[link] = (old, reserved)
        yield
        if w.head == old:
            w.head = link + 1
            return
        yield


def await_group(w, promises):
    m = len(promises)
    if w.sem == 0:                         # released already: pass straight on
        w.out.extend(promises)
        return
    yield
    fresh, dst, base = None, None, None
    while dst is None:
        old = w.partial
        yield
        tag, c, l1 = old
        if l1 and c + m <= SLOTS:
            if w.cas_partial(old, (tag + 1, c + m, l1)):
                dst, base = l1 - 1, c
            continue
        if fresh is None:
            fresh = w.free.pop(0)
            w.written[fresh] = 0
            w.slots[fresh] = {}
            yield
        if w.cas_partial(old, (tag + 1, m, fresh + 1)):
            dst, base, fresh = fresh, 0, None
            if l1:
                yield from retire(w, l1 - 1, c)
    if fresh is not None:
        w.free.append(fresh)
    for r, p in enumerate(promises):       # each lane writes its slot
        assert base + r < SLOTS
        w.slots[dst][base + r] = p
        yield
    w.written[dst] += m
    yield
    if w.sem == 0:                         # released meanwhile: sweep for ourselves
        yield from sweep(w)


def decrement(w, n):
    w.sem -= n
    yield
    if w.sem == 0:
        yield from sweep(w)


def consumer(w, rng):
    # takes published links and frees them, so that links are reused (ABA on the partial word)
    while True:
        if w.queue and rng.random() < 0.5:
            link = w.queue.pop(0)
            w.free.append(link)
        yield


def run(seed):
    rng = random.Random(seed)
    groups = []
    pid = 0
    for _ in range(rng.randint(1, 40)):
        m = rng.randint(1, 32)
        groups.append(list(range(pid, pid + m)))
        pid += m
    n_dec = rng.randint(1, 8)
    w = World(n_links=4 * len(groups) + 8, sem=n_dec)
    # Awaiting groups and the decrements that release the barrier run concurrently, so a
    # release can come while groups are between their reservation and their writes (the
    # barrier demo, where each group decrements after its own await, is one such order).
    def member(g, dec):
        yield from await_group(w, g)
        if dec:
            yield from decrement(w, 1)
    late = [list(range(pid + 100 * k, pid + 100 * k + rng.randint(1, 5))) for k in range(rng.randint(0, 3))]
    if rng.random() < 0.5:
        actors = [await_group(w, g) for g in groups] + [decrement(w, 1) for _ in range(n_dec)]
    else:
        w.sem = len(groups)
        actors = [member(g, True) for g in groups]
    cons = consumer(w, rng)
    steps = 0
    while actors:
        a = rng.choice(actors)
        try:
            next(a)
        except StopIteration:
            actors.remove(a)
        if rng.random() < 0.2:
            next(cons)
        steps += 1
        assert steps < 10 ** 6
    for g in late:  # arrive after the release: passed straight on
        for _ in await_group(w, g):
            pass
    expected = sorted(p for g in groups + late for p in g)
    return sorted(w.out), expected, w


def test_every_held_promise_comes_out_exactly_once():
    for seed in range(1500):
        got, expected, w = run(seed)
        assert got == expected, seed
        assert w.partial[2] == 0 and w.head == 0, seed  # nothing left held after the release
