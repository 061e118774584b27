"""Model check of the tensor-core pipeline's mbarrier protocol (CPU).

The pipeline of cp-paw_b200/csrc/tc_pipe.cuh hands every chunk through six
kinds of mbarriers (rawfull, rawempty, sfull, sfree, bfull, bempty) between
a copy warp, a split-B copy warp, two groups of converter warps, the MMA
thread and the drain warps.  A waiter passes a parity wait when the barrier's
current phase parity differs from the parity it asks for, so a role that runs
two phases ahead of a barrier passes on the wrong phase.  This test replays
the protocol of every pipe configuration declared in tc.cu under random
interleavings of the roles and of the asynchronous events (copies landing in
any order, MMA groups completing in issue order) and checks that every role
reads the data of its own chunk, that nothing overwrites data still in use
and that the run never deadlocks.  No reference counterpart: the reference
computes these products with BLAS on the host."""

import pathlib
import random
import re

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
TC = ROOT / "cp-paw_b200" / "csrc" / "tc.cu"


class Bar:
    """mbarrier: arrival count, transaction count, phase number."""

    def __init__(self, count):
        self.count = count
        self.pending = count
        self.tx = 0
        self.phase = 0

    def arrive(self, expect_tx=0):
        self.tx += expect_tx
        self.pending -= 1
        self._complete()

    def complete_tx(self, n):
        self.tx -= n
        self._complete()

    def _complete(self):
        assert self.pending >= 0, "more arrivals than the barrier's count"
        if self.pending == 0 and self.tx == 0:
            self.phase += 1
            self.pending = self.count

    def passes(self, parity):
        return (self.phase & 1) != parity


class Violation(Exception):
    pass


def check(cond, what):
    if not cond:
        raise Violation(what)


def simulate(nsplit, nraw, bpre, cpr, nreg, nchunk, seed, conv_warps=2, drain_warps=2):
    """One random interleaving; raises Violation on a protocol error."""
    rng = random.Random(seed)
    rawfull = [Bar(1) for _ in range(nraw)]
    # the warps of one converter group (conv_warps of them) all arrive for the
    # group's chunk
    rawempty = [Bar(conv_warps) for _ in range(nraw)]
    sfull = [Bar(conv_warps + (1 if bpre else 0)) for _ in range(nsplit)]
    sfree = [Bar(1) for _ in range(nsplit)]
    bfull = [Bar(1) for _ in range(nreg)]
    bempty = [Bar(drain_warps) for _ in range(nreg)]
    raw = [None] * nraw
    sa = [None] * nsplit
    sb = [None] * nsplit
    region = [None] * nreg
    drained = [-1] * drain_warps
    copies = []  # landing events, any order
    mmas = []  # completion events, issue order
    nregions = (nchunk + cpr - 1) // cpr

    def land_raw(slot, c):
        raw[slot] = c
        rawfull[slot].complete_tx(1)

    def land_b(s, c):
        sb[s] = c
        sfull[s].complete_tx(1)

    def copy_a():
        for c in range(nchunk):
            slot = c % nraw
            if c >= nraw:
                yield rawempty[slot], ((c // nraw) - 1) & 1
            copies.append((land_raw, slot, c))
            yield None
            rawfull[slot].arrive(expect_tx=1)

    def copy_b():
        for c in range(nchunk):
            s = c % nsplit
            if c >= nsplit:
                yield sfree[s], ((c // nsplit) - 1) & 1
            copies.append((land_b, s, c))
            yield None
            sfull[s].arrive(expect_tx=1)

    def converter(grp):
        for c in range(grp, nchunk, 2):
            s, slot = c % nsplit, c % nraw
            yield rawfull[slot], (c // nraw) & 1
            if c >= nsplit:
                yield sfree[s], ((c // nsplit) - 1) & 1
            check(raw[slot] == c, f"converter of chunk {c} reads raw slot {slot} holding {raw[slot]}")
            yield None
            sa[s] = c
            if not bpre:
                sb[s] = c
            check(raw[slot] == c, f"raw slot {slot} overwritten while chunk {c} converts")
            sfull[s].arrive()
            rawempty[slot].arrive()

    def mma():
        for u in range(nregions):
            r, c0 = u % nreg, u * cpr
            nc = min(cpr, nchunk - c0)
            if u >= nreg:
                yield bempty[r], ((u // nreg) - 1) & 1
            check(all(d >= u - nreg for d in drained), f"region {u} issued before region {u - nreg} drained")
            for i in range(nc):
                c = c0 + i
                yield sfull[c % nsplit], (c // nsplit) & 1
            for i in range(nc):
                c = c0 + i
                s = c % nsplit
                check(sa[s] == c and sb[s] == c, f"MMA of chunk {c} issued on stage {s} holding {sa[s]}/{sb[s]}")
            mmas.append(u)
            yield None

    def mma_done(u):
        r, c0 = u % nreg, u * cpr
        nc = min(cpr, nchunk - c0)
        for i in range(nc):
            c = c0 + i
            s = c % nsplit
            check(sa[s] == c and sb[s] == c, f"stage {s} overwritten before the MMA of chunk {c} completed")
        region[r] = u
        bfull[r].arrive()
        for i in range(nc):
            sfree[(c0 + i) % nsplit].arrive()

    def drain(w):
        for u in range(nregions):
            r = u % nreg
            yield bfull[r], (u // nreg) & 1
            check(region[r] == u, f"drain of region {u} reads {region[r]}")
            yield None
            check(region[r] == u, f"region {u} overwritten while drained")
            drained[w] = u
            bempty[r].arrive()

    actors = [copy_a(), mma()]
    if bpre:
        actors.append(copy_b())
    for _ in range(conv_warps):
        actors.append(converter(0))
        actors.append(converter(1))
    for w in range(drain_warps):
        actors.append(drain(w))
    state = {a: next(a, "done") for a in actors}
    while True:
        live = [a for a, w in state.items() if w != "done"]
        ready = [a for a in live if state[a] is None or state[a][0].passes(state[a][1])]
        choices = [("actor", a) for a in ready] + [("copy", i) for i in range(len(copies))]
        if mmas:
            choices.append(("mma", 0))
        if not choices:
            check(not live, f"deadlock with {len(live)} roles waiting")
            break
        kind, x = rng.choice(choices)
        if kind == "actor":
            state[x] = next(x, "done")
        elif kind == "copy":
            fn, *args = copies.pop(x)
            fn(*args)
        else:
            mma_done(mmas.pop(0))
    check(drained == [nregions - 1] * drain_warps, "not every region drained")


def pipe_configs():
    src = TC.read_text()
    consts = dict(re.findall(r"\b(k\w+) = (\d+)", src))
    out = {}
    for name, args in re.findall(r"using (\w+) = tc::Pipe<([^>]*)>;", src):
        vals = []
        for a in (x.strip() for x in args.split(",")):
            if a in ("true", "false"):
                vals.append(int(a == "true"))
            else:
                vals.append(int(consts.get(a, a)))
        nsplit, nraw = vals[0], vals[1]
        bpre = bool(vals[3]) if len(vals) > 3 else True
        cpr = vals[4] if len(vals) > 4 else 2
        nreg = vals[5] if len(vals) > 5 else 2
        out[name] = (nsplit, nraw, bpre, cpr, nreg)
    return out


CONFIGS = pipe_configs()
NCHUNKS = (1, 2, 3, 4, 5, 7, 9, 16, 23, 40)


def test_configs_found():
    assert {"ProjPipe", "AddproPipe", "GramPipe", "AddxPipe", "ForcePipe", "GemmPipe"} <= set(CONFIGS)


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_protocol_holds_under_random_interleavings(name):
    nsplit, nraw, bpre, cpr, nreg = CONFIGS[name]
    for nchunk in NCHUNKS:
        for seed in range(40):
            simulate(nsplit, nraw, bpre, cpr, nreg, nchunk, seed)


def test_model_finds_an_odd_raw_slot_count():
    """Planted mistake in the model: three raw slots shared by the two
    converter groups let a group pass a parity wait one phase early."""
    found = False
    for seed in range(400):
        try:
            simulate(8, 3, True, 2, 2, 40, seed)
        except Violation:
            found = True
            break
    assert found
