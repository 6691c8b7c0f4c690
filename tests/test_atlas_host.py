"""CPU-sourced atlas sync on the CPU: r3d_host_atlas_pick against a Python
restatement of the reference's two-pass round (src/vk/vkbackend.c:4990-5060:
stale slots zeroed first, then slots whose brick's content generation
changed, at most the budget, in slot order) over a scripted run of slot
reassignments, generation bumps and budgets, with each round's picks
applied to the keys; and brick location from the page table."""
import ctypes as C
import math

import numpy as np

ABSENT = 0xFFFFFFFF


def _page(shape=(700, 600, 300), nlev=3):
    off, levels = 64, []
    for li in range(nlev):
        s = 128 << li
        bd = [(n + s - 1) // s for n in shape]
        levels.append((off, bd[0] | (bd[1] << 10) | (bd[2] << 20), 1 << li, bd))
        off += math.prod(bd)
    page = np.full(off, ABSENT, np.uint32)
    page[:64] = 0
    page[0], page[1:4] = nlev, shape
    for li, (o, pk, sc, _) in enumerate(levels):
        page[4 + 4 * li:7 + 4 * li] = (o, pk, sc)
    return page, levels


def _locate(levels, b):
    for li, (o, _, _, bd) in enumerate(levels):
        if o <= b < o + math.prod(bd):
            loc = b - o
            return li, loc % bd[0], (loc // bd[0]) % bd[1], loc // (bd[0] * bd[1])
    raise AssertionError(b)


def _pick_ref(levels, slot_brick, keys, gen, budget):
    budget = 16 if budget == 0 or budget > 16 else budget
    out = []
    for s, b in enumerate(slot_brick):
        if len(out) >= budget:
            break
        if b == ABSENT:
            continue
        k = int(keys[s])
        if k == 0 or (k >> 32) == b + 1:
            continue
        out.append((s, b, 0))
    if out:
        return out
    for s, b in enumerate(slot_brick):
        if len(out) >= budget:
            break
        if b == ABSENT:
            continue
        g = gen(*_locate(levels, int(b)))
        want = ((int(b) + 1) << 32 | g) if g else 0
        if int(keys[s]) == want:
            continue
        out.append((s, int(b), want))
    return out


def test_brick_locate(rb):
    page, levels = _page()
    for b in (64, 65, 64 + 6 * 5 * 3 - 1, levels[1][0], levels[2][0] + 3, len(page) - 1):
        lv = [C.c_uint32() for _ in range(4)]
        assert rb.lib.r3d_host_brick_locate(page.ctypes.data, b, *[C.byref(x) for x in lv]) == 0
        assert tuple(x.value for x in lv) == _locate(levels, b)
    lv = [C.c_uint32() for _ in range(4)]
    assert rb.lib.r3d_host_brick_locate(page.ctypes.data, len(page), *[C.byref(x) for x in lv]) != 0


def test_atlas_pick_matches_restatement(rb):
    page, levels = _page()
    nb = len(page) - 64
    rng = np.random.default_rng(17)
    nslots = 40
    slot_brick = np.full(nslots, ABSENT, np.uint32)
    slot_brick[:30] = 64 + rng.choice(nb, 30, replace=False)
    keys = np.zeros(nslots, np.uint64)
    gens = {}  # brick -> generation (absent: 1 for even bricks, 0 for odd)

    def gen(l, x, y, z):
        b = levels[l][0] + (z * levels[l][3][1] + y) * levels[l][3][0] + x
        return gens.get(b, 1 if b % 2 == 0 else 0)

    src = rb.brick_src(gen, lambda *a: np.zeros(128 ** 3, np.uint8))
    sel = (C.c_uint32 * 16)()
    selb = (C.c_uint32 * 16)()
    selk = (C.c_uint64 * 16)()
    rounds = 0
    for step in range(60):
        if step % 7 == 3:  # the pump reassigns a few slots
            for s in rng.choice(nslots, 5, replace=False):
                slot_brick[s] = 64 + rng.integers(nb) if rng.random() < 0.8 else ABSENT
        if step % 5 == 1:  # paint strokes: generations move
            for b in rng.choice(slot_brick[slot_brick != ABSENT], 3):
                gens[int(b)] = gens.get(int(b), 1) + 1
        if step % 11 == 6:  # a source with no content for some bricks
            gens[int(slot_brick[0])] = 0
        budget = [0, 3, 16, 40, 1][step % 5]
        want = _pick_ref(levels, slot_brick, keys, gen, budget)
        n = rb.lib.r3d_host_atlas_pick(page.ctypes.data, slot_brick.ctypes.data, nslots,
                                       keys.ctypes.data, C.byref(src), budget, sel, selb, selk)
        got = [(sel[i], selb[i], selk[i]) for i in range(n)]
        assert got == want, step
        for s, _, k in got:
            keys[s] = k
        rounds += bool(n)
    assert rounds > 20
    # a settled atlas picks nothing
    for _ in range(10):
        n = rb.lib.r3d_host_atlas_pick(page.ctypes.data, slot_brick.ctypes.data, nslots,
                                       keys.ctypes.data, C.byref(src), 16, sel, selb, selk)
        for i in range(n):
            keys[sel[i]] = selk[i]
    assert rb.lib.r3d_host_atlas_pick(page.ctypes.data, slot_brick.ctypes.data, nslots,
                                      keys.ctypes.data, C.byref(src), 16, sel, selb, selk) == 0
