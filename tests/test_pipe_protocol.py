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


def simulate(nsplit, nraw, bpre, cpr, nreg, nchunk, seed, conv_warps=2, drain_warps=2, g=1):
    """One random interleaving; raises Violation on a protocol error.  g
    chunks travel together as one unit through a raw slot and a stage (each
    of g chunk places), with one hand-over per unit."""
    rng = random.Random(seed)
    rawfull = [Bar(1) for _ in range(nraw)]
    # the warps of one converter group (conv_warps of them) all arrive for the
    # group's chunk
    rawempty = [Bar(conv_warps) for _ in range(nraw)]
    sfull = [Bar(conv_warps + (1 if bpre else 0)) for _ in range(nsplit)]
    sfree = [Bar(1) for _ in range(nsplit)]
    bfull = [Bar(1) for _ in range(nreg)]
    bempty = [Bar(drain_warps) for _ in range(nreg)]
    raw = [None] * (nraw * g)
    sa = [None] * (nsplit * g)
    sb = [None] * (nsplit * g)
    region = [None] * nreg
    drained = [-1] * drain_warps
    copies = []  # landing events, any order
    mmas = []  # completion events, issue order
    nregions = (nchunk + cpr - 1) // cpr
    nunits = (nchunk + g - 1) // g
    assert cpr % g == 0

    def chunks(q):
        return range(q * g, min(nchunk, (q + 1) * g))

    def place(q, c, n):  # chunk c's place in the slot or stage of unit q (n of them)
        return (q % n) * g + c - q * g

    def land_raw(i, c):
        raw[i] = c
        rawfull[i // g].complete_tx(1)

    def land_b(i, c):
        sb[i] = c
        sfull[i // g].complete_tx(1)

    def copy_a():
        for q in range(nunits):
            slot = q % nraw
            if q >= nraw:
                yield rawempty[slot], ((q // nraw) - 1) & 1
            for c in chunks(q):
                copies.append((land_raw, place(q, c, nraw), c))
            yield None
            rawfull[slot].arrive(expect_tx=len(chunks(q)))

    def copy_b():
        for q in range(nunits):
            s = q % nsplit
            if q >= nsplit:
                yield sfree[s], ((q // nsplit) - 1) & 1
            for c in chunks(q):
                copies.append((land_b, place(q, c, nsplit), c))
            yield None
            sfull[s].arrive(expect_tx=len(chunks(q)))

    def converter(grp):
        for q in range(grp, nunits, 2):
            s, slot = q % nsplit, q % nraw
            yield rawfull[slot], (q // nraw) & 1
            if q >= nsplit:
                yield sfree[s], ((q // nsplit) - 1) & 1
            for c in chunks(q):
                i = place(q, c, nraw)
                check(raw[i] == c, f"converter of chunk {c} reads raw place {i} holding {raw[i]}")
            yield None
            for c in chunks(q):
                sa[place(q, c, nsplit)] = c
                if not bpre:
                    sb[place(q, c, nsplit)] = c
                i = place(q, c, nraw)
                check(raw[i] == c, f"raw place {i} overwritten while chunk {c} converts")
            sfull[s].arrive()
            rawempty[slot].arrive()

    def units(u):  # the units of region u
        c0 = u * cpr
        return range(c0 // g, (min(nchunk, c0 + cpr) + g - 1) // g)

    def mma():
        for u in range(nregions):
            r, c0 = u % nreg, u * cpr
            nc = min(cpr, nchunk - c0)
            if u >= nreg:
                yield bempty[r], ((u // nreg) - 1) & 1
            check(all(d >= u - nreg for d in drained), f"region {u} issued before region {u - nreg} drained")
            for q in units(u):
                yield sfull[q % nsplit], (q // nsplit) & 1
            for c in range(c0, c0 + nc):
                s = place(c // g, c, nsplit)
                check(sa[s] == c and sb[s] == c, f"MMA of chunk {c} issued on stage place {s} holding {sa[s]}/{sb[s]}")
            mmas.append(u)
            yield None

    def mma_done(u):
        r, c0 = u % nreg, u * cpr
        nc = min(cpr, nchunk - c0)
        for c in range(c0, c0 + nc):
            s = place(c // g, c, nsplit)
            check(sa[s] == c and sb[s] == c, f"stage place {s} overwritten before the MMA of chunk {c} completed")
        region[r] = u
        bfull[r].arrive()
        for q in units(u):
            sfree[q % nsplit].arrive()

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
        g = vals[6] if len(vals) > 6 else 1
        out[name] = (nsplit, nraw, bpre, cpr, nreg, g)
    return out


CONFIGS = pipe_configs()
NCHUNKS = (1, 2, 3, 4, 5, 7, 9, 16, 23, 40)


def test_configs_found():
    assert {"ProjPipe", "AddproPipe", "GramPipe", "AddxPipe", "ForcePipe", "GemmPipe"} <= set(CONFIGS)


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_protocol_holds_under_random_interleavings(name):
    nsplit, nraw, bpre, cpr, nreg, g = CONFIGS[name]
    for nchunk in NCHUNKS:
        for seed in range(40):
            simulate(nsplit, nraw, bpre, cpr, nreg, nchunk, seed, g=g)


@pytest.mark.parametrize("nsplit,nraw,cpr,g", [(4, 4, 2, 2), (4, 2, 4, 2), (2, 4, 4, 4)])
def test_protocol_holds_with_units_of_several_chunks(nsplit, nraw, cpr, g):
    for nchunk in NCHUNKS:
        for seed in range(20):
            simulate(nsplit, nraw, True, cpr, 2, nchunk, seed, g=g)


def test_model_finds_an_odd_raw_slot_count():
    """Planted mistake in the model: three raw slots shared by the two
    converter groups let a group pass a parity wait one phase early."""
    for g in (1, 2):
        found = False
        for seed in range(400):
            try:
                simulate(8 // g, 3, True, 2, 2, 40, seed, g=g)
            except Violation:
                found = True
                break
        assert found, g


def simulate_force(nchk, w0, w1, tn, nstage, seed, conv_warps=2, drain_warps=2, plant=None):
    """Protocol of the persistent force kernel (k_tc_force_p): items
    (g tile m, projector tile n) = divmod(w, tn) for w in [w0, w1); the A tile
    (all nchk chunks) stays resident while the items of one m run; two raw
    slots, per-chunk afull barriers, one afree barrier, nstage B stages, two
    accumulation regions holding one item each."""
    rng = random.Random(seed)
    m_first = w0 // tn
    nm = (w1 - 1) // tn - m_first + 1
    rpi = nchk // 2
    rawfull = [Bar(1) for _ in range(2)]
    rawempty = [Bar(conv_warps) for _ in range(2)]
    afull = [Bar(conv_warps) for _ in range(nchk)]
    afree = Bar(1)
    sfull = [Bar(1) for _ in range(nstage)]
    sfree = [Bar(1) for _ in range(nstage)]
    bfull = [Bar(1) for _ in range(2)]
    bempty = [Bar(drain_warps) for _ in range(2)]
    raw = [None, None]
    atile = [None] * nchk
    stage = [None] * nstage
    region = [None, None]
    copies, mmas = [], []

    def land(kind, idx, val):
        if kind == "raw":
            raw[idx] = val
            rawfull[idx].complete_tx(1)
        else:
            stage[idx] = val
            sfull[idx].complete_tx(1)

    def copy_a():
        for q in range(nm * nchk):
            slot = q & 1
            if q >= 2:
                yield rawempty[slot], ((q >> 1) - 1) & 1
            copies.append(("raw", slot, q))
            yield None
            rawfull[slot].arrive(expect_tx=1)

    def copy_b():
        j = 0
        for w in range(w0, w1):
            for c in range(nchk):
                s = j % nstage
                if j >= nstage:
                    yield sfree[s], ((j // nstage) - 1) & 1
                copies.append(("stage", s, (w, c)))
                yield None
                sfull[s].arrive(expect_tx=1)
                j += 1

    def converter(grp):
        for im in range(nm):
            for c in range(grp, nchk, 2):
                q = im * nchk + c
                slot = q & 1
                yield rawfull[slot], (q >> 1) & 1
                if c == grp and im >= 1 and plant != "no_afree":
                    yield afree, (im - 1) & 1
                check(raw[slot] == q, f"converter of A chunk {q} reads slot holding {raw[slot]}")
                yield None
                atile[c] = im
                check(raw[slot] == q, f"raw slot {slot} overwritten during conversion of {q}")
                afull[c].arrive()
                rawempty[slot].arrive()

    drained = [-1] * drain_warps

    def mma():
        it = j = 0
        for w in range(w0, w1):
            im = w // tn - m_first
            first = w == w0 or w % tn == 0
            last = w == w1 - 1 or (w + 1) % tn == 0
            r = it & 1
            if it >= 2:
                yield bempty[r], ((it >> 1) - 1) & 1
            check(all(d >= it - 2 for d in drained), f"item {it} written before item {it - 2} was drained")
            for rr in range(rpi):
                for i in range(2):
                    if first:
                        yield afull[2 * rr + i], im & 1
                    yield sfull[(j + i) % nstage], ((j + i) // nstage) & 1
                for i in range(2):
                    c = 2 * rr + i
                    check(atile[c] == im, f"MMA of item {w} chunk {c}: A holds tile {atile[c]}")
                    check(stage[(j + i) % nstage] == (w, c), f"MMA of item {w} chunk {c}: stage holds wrong chunk")
                mmas.append(("pair", w, rr, j, im))
                yield None
                j += 2
            mmas.append(("item", it, last))
            it += 1

    def mma_done(kind, *a):
        if kind == "pair":
            w, rr, j, im = a
            for i in range(2):
                c = 2 * rr + i
                check(atile[c] == im, f"A chunk {c} overwritten before the MMA of item {w} completed")
                check(stage[(j + i) % nstage] == (w, c), f"stage overwritten before the MMA of item {w} completed")
            sfree[j % nstage].arrive()
            sfree[(j + 1) % nstage].arrive()
        else:
            it, last = a
            region[it & 1] = it
            bfull[it & 1].arrive()
            if last:
                afree.arrive()

    def drain(k):
        for it in range(w1 - w0):
            r = it & 1
            yield bfull[r], (it >> 1) & 1
            check(region[r] == it, f"drain of item {it} reads {region[r]}")
            yield None
            check(region[r] == it, f"region of item {it} overwritten while read")
            drained[k] = it
            bempty[r].arrive()

    actors = [copy_a(), copy_b(), mma()]
    for _ in range(conv_warps):
        actors += [converter(0), converter(1)]
    actors += [drain(k) for k in range(drain_warps)]
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
            land(*copies.pop(x))
        else:
            mma_done(*mmas.pop(0))


def force_stages():
    m = re.search(r"constexpr int kFNS = (\d+);", TC.read_text())
    assert m
    return int(m.group(1))


@pytest.mark.parametrize("nchk", [2, 4, 8])
def test_force_protocol_holds_under_random_interleavings(nchk):
    ns = force_stages()
    for (w0, w1, tn) in [(0, 10, 8), (5, 17, 8), (3, 4, 2), (0, 9, 1), (7, 30, 4)]:
        for seed in range(25):
            simulate_force(nchk, w0, w1, tn, ns, seed)


def test_force_model_finds_a_missing_afree_wait():
    """Planted mistake in the model: converters that do not wait for the MMAs
    of the previous g tile overwrite its resident A operand."""
    found = False
    for seed in range(300):
        try:
            simulate_force(4, 0, 12, 2, force_stages(), seed, plant="no_afree")
        except Violation:
            found = True
            break
    assert found
