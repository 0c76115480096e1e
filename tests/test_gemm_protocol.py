"""CPU check of the barrier protocol of the persistent tcgen05 GEMM (csrc/cnn_gemm.cu,
umma_gemm_kernel): one producer lane (TMA stage fills), one MMA lane (stage reads into one of
two TMEM accumulators per tile) and four epilogue warps (accumulator read-back), coupled only
by mbarriers with phase parities.  The roles are stepped in random orders, the TMA loads land
and the MMAs complete at random later times (the MMAs in issue order), and the test checks
that every CTA finishes (no deadlock), that no stage is refilled before the MMAs that read it
completed, that the MMAs read each stage fill of their own tile and K block, and that the
epilogue reads each tile's finished accumulator and no accumulator is rewritten before all
four epilogue warps released it.  The tile decoding and the parities are the kernel's."""
import random

import pytest

STAGES = 4


class Bar:
    """An mbarrier: `count` arrivals complete a phase; try_wait.parity(p) succeeds when the
    phase of parity p has completed (the current phase's parity differs from p)."""

    def __init__(self, count):
        self.count, self.pending, self.completed = count, count, 0

    def arrive(self):
        self.pending -= 1
        if self.pending == 0:
            self.completed += 1
            self.pending = self.count

    def ok(self, parity):
        return (self.completed & 1) != parity


def _simulate_cta(tiles, kb_range, rnd):
    full = [Bar(1) for _ in range(STAGES)]
    empty = [Bar(1) for _ in range(STAGES)]
    acc_full, acc_empty = [Bar(1), Bar(1)], [Bar(4), Bar(4)]
    stage = [None] * STAGES          # (tile, kb, state) of each stage's current fill
    acc = [None, None]               # tile whose MMAs completed in each accumulator
    landing, mma_queue = [], []      # pending TMA completions; MMA completions in order
    prod = {"ti": 0, "kb": None, "it": 0}
    mma = {"ti": 0, "kb": None, "it": 0, "tc": 0, "open": False}
    epi = [{"ti": 0, "tc": 0} for _ in range(4)]

    def producer():
        if prod["ti"] >= len(tiles):
            return False
        t = tiles[prod["ti"]]
        kb0, kb1 = kb_range(t)
        if prod["kb"] is None:
            prod["kb"] = kb0
        it = prod["it"]
        s = it % STAGES
        if it >= STAGES and not empty[s].ok(((it // STAGES) - 1) & 1):
            return False
        assert stage[s] is None or stage[s][2] == "read", ("refilled before its MMAs completed", stage[s])
        stage[s] = (t, prod["kb"], "loading")

        def land(s=s, t=t, kb=prod["kb"]):
            stage[s] = (t, kb, "full")
            full[s].arrive()

        landing.append(land)
        prod["it"] += 1
        prod["kb"] += 1
        if prod["kb"] >= kb1:
            prod["ti"] += 1
            prod["kb"] = None
        return True

    def mma_lane():
        if mma["ti"] >= len(tiles):
            return False
        t = tiles[mma["ti"]]
        kb0, kb1 = kb_range(t)
        b = mma["tc"] & 1
        if not mma["open"]:
            if mma["tc"] >= 2 and not acc_empty[b].ok(((mma["tc"] >> 1) - 1) & 1):
                return False
            assert acc[b] is None, ("accumulator rewritten before its epilogue", acc[b])
            mma["open"], mma["kb"] = True, kb0
        it = mma["it"]
        s = it % STAGES
        if not full[s].ok((it // STAGES) & 1):
            return False
        assert stage[s] == (t, mma["kb"], "full"), ("MMA read the wrong fill", stage[s], t, mma["kb"])
        stage[s] = (t, mma["kb"], "reading")

        def read_done(s=s):
            stage[s] = stage[s][:2] + ("read",)
            empty[s].arrive()

        mma_queue.append(read_done)
        mma["it"] += 1
        mma["kb"] += 1
        if mma["kb"] >= kb1:
            def acc_done(b=b, t=t):
                acc[b] = t
                acc_full[b].arrive()

            mma_queue.append(acc_done)
            mma["ti"] += 1
            mma["tc"] += 1
            mma["open"] = False
        return True

    def epilogue(w):
        e = epi[w]
        if e["ti"] >= len(tiles):
            return False
        t = tiles[e["ti"]]
        b = e["tc"] & 1
        if not acc_full[b].ok((e["tc"] >> 1) & 1):
            return False
        assert acc[b] == t, ("epilogue read the wrong accumulator", acc[b], t)
        acc_empty[b].arrive()
        if acc_empty[b].pending == 4:  # all four warps released it
            acc[b] = None
        e["ti"] += 1
        e["tc"] += 1
        return True

    roles = [producer, mma_lane] + [lambda w=w: epilogue(w) for w in range(4)]
    for _ in range(200000):
        rnd.shuffle(roles)
        for r in roles:
            if rnd.random() < 0.5:
                r()
        if landing and rnd.random() < 0.5:
            landing.pop(rnd.randrange(len(landing)))()
        if mma_queue and rnd.random() < 0.5:
            mma_queue.pop(0)()
        if (prod["ti"] >= len(tiles) and mma["ti"] >= len(tiles) and all(e["ti"] >= len(tiles) for e in epi)
                and not landing and not mma_queue):
            return
    raise AssertionError("deadlock")


@pytest.mark.parametrize("seed", range(60))
def test_persistent_gemm_protocol(seed):
    rnd = random.Random(seed)
    tiles_m, tiles_n, splits = rnd.randint(1, 9), rnd.randint(1, 4), rnd.randint(1, 3)
    kb_total = rnd.randint(splits, 20)
    per = (kb_total + splits - 1) // splits
    splits = (kb_total + per - 1) // per  # as the launcher: every split holds a K block
    ntiles = tiles_m * tiles_n * splits
    grid = rnd.randint(1, ntiles)

    def kb_range(t):  # TileGrid::decode
        sp = (t // tiles_n) // tiles_m
        return sp * per, min(kb_total, sp * per + per)

    for cta in range(grid):
        _simulate_cta(list(range(cta, ntiles, grid)), kb_range, rnd)
