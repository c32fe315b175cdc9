"""The served form (stormgpu_server_*): a resident three-step -O seed chain serving batches of
mixed read lengths.  Every batch's results must equal the plain path run step by step (map with
the first seed family, keep the reads it left unmapped, map those with the next one: the
reference re-run on its own -O output), both when the batch runs alone and when all batches are
submitted together from several threads and overlap on the GPU."""
import threading

import numpy as np
import pytest

import ffi
from storm_b200 import api, synth

pytestmark = pytest.mark.gpu

CHAIN = ["###-##--#-##-#-###", "####-#-#--##-###", "#####-##-###"]
ARGS = dict(indels=15, min_score=100, min_score_filter=100)


def _pack_batch(seqs, quals):
    n = len(seqs)
    L = max(len(s) for s in seqs)
    stride = ((L + 3) // 4 + 15) & ~7
    codes = np.zeros((n, stride), np.uint8)
    levels = np.zeros((n, stride), np.uint8)
    for i, (s, q) in enumerate(zip(seqs, quals)):
        p = ffi.pack2(s)
        codes[i, :len(p)] = p
        lv = ffi.pack2(np.searchsorted(np.array([2, 7, 10]), np.asarray(q), side="left"))
        levels[i, :len(lv)] = lv
    lengths = np.array([len(s) for s in seqs], np.int16)
    return api.ReadBatch(codes, lengths, levels)


@pytest.fixture(scope="module")
def world():
    genome = synth.make_genome([250000, 60000], 33, 0.41, 0.3)
    refs = []
    for _, seq in genome:
        cp = ffi.pack2(seq, 1024)
        mk = ffi.pack2(np.zeros(len(seq), np.uint8), 1024, fill=0x55)
        refs.append((cp, mk, len(seq)))
    batches = []
    rng = np.random.default_rng(77)
    hard = synth.ReadModel(sub_lo=0.08, sub_hi=0.14, indel_rate=0.004, indel_max=2)
    for k, n in enumerate([40, 700, 2500, 1200, 9]):
        seqs, quals = synth.simulate_nucleotide_reads(genome, n, [35, 50, 75, 100], 100 + k)
        hs, hq = synth.simulate_nucleotide_reads(genome, n, [50, 75, 100], 200 + k, hard)
        seqs, quals = list(seqs) + list(hs), list(quals) + list(hq)
        for _ in range(max(1, n // 20)):  # reads from nowhere: no step maps them
            L = int(rng.choice([35, 50, 75]))
            seqs.append(rng.integers(0, 4, size=L).astype(np.uint8))
            quals.append(np.full(L, 30, np.int64))
        order = rng.permutation(len(seqs))
        batches.append(_pack_batch([seqs[i] for i in order], [quals[i] for i in order]))
    return genome, refs, batches


def _add(target, refs):
    for cp, mk, n in refs:
        target.add_reference(cp[1024:], mk[1024:], n)


def _plain_chain(refs, batch, tbs):
    prm = api.params(**ARGS)
    n = batch.n
    hits = np.zeros(n * 4, dtype=api.HIT_DTYPE)
    hits["ref_id"] = -1
    tb = np.zeros((n * 4, tbs), np.uint8)
    mapped = np.zeros(n, np.uint8)
    step = np.full(n, 255, np.uint8)
    ids = np.arange(n)
    cur = batch
    for k, seeds in enumerate(CHAIN):
        if cur.n == 0:
            break
        m = api.Mapper(prm, seeds)
        _add(m, refs)
        m.build_index()
        res = m.map(cur, tbs)
        m.close()
        got = res.mapped != 0
        for j in np.nonzero(got)[0]:
            o = ids[j]
            hits[4 * o:4 * o + 4] = res.hits[4 * j:4 * j + 4]
            tb[4 * o:4 * o + 4] = res.tb[4 * j:4 * j + 4]
            mapped[o] = 1
            step[o] = k
        keep = np.nonzero(~got)[0]
        ids = ids[keep]
        cur = api.ReadBatch(cur.codes[keep], cur.lengths[keep], cur.levels[keep])
    return hits, tb, mapped, step


def _same(served, plain, ctx):
    res, step, _ = served
    hits, tb, mapped, pstep = plain
    assert np.array_equal(res.mapped != 0, mapped != 0), ctx
    assert np.array_equal(step, pstep), ctx
    live = np.repeat(mapped != 0, 4)
    assert res.hits[live].tobytes() == hits[live].tobytes(), ctx
    for i in np.nonzero(live)[0]:
        nb = (int(hits["tb_len"][i]) + 1) // 2
        assert bytes(res.tb[i, :nb]) == bytes(tb[i, :nb]), (ctx, i)


def test_served_chain_equals_plain_chain_alone_and_in_the_mix(world):
    _, refs, batches = world
    tbs = ((100 + ARGS["indels"] + 1) // 2 + 7) & ~7
    plain = [_plain_chain(refs, b, tbs) for b in batches]
    assert sum(int(p[2].sum()) for p in plain) > 1000
    steps = {int(s) for p in plain for s in p[3]}
    assert {0, 1, 255} <= steps, steps  # reads mapped at several steps, and some at none
    srv = api.Server(api.params(**ARGS), CHAIN, slots=3, budget_bytes=2 << 30)
    _add(srv, refs)
    # launch parameters other than the plain chain's: they must change no result
    srv.set_tuning(gather_warp_cap=1536, gather_reads_per_steal=1, filter_cursor=1, filter_rows=2, align_steal=64)
    srv.build()
    with pytest.raises(api.StormError, match="before"):
        srv.set_tuning()
    for i, b in enumerate(batches):  # alone
        t = srv.submit(b, tbs)
        _same(srv.poll(t), plain[i], ("alone", i))
    tickets = [None] * len(batches)

    def go(i):
        tickets[i] = srv.submit(batches[i], tbs)
    ths = [threading.Thread(target=go, args=(i,)) for i in range(len(batches))]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    for i, t in enumerate(tickets):  # in the mix
        out = srv.poll(t)
        assert out[2] > 0
        _same(out, plain[i], ("mix", i))
    srv.close()


def test_server_rejects_a_batch_beyond_its_budget(world):
    _, refs, batches = world
    srv = api.Server(api.params(**ARGS), CHAIN[:1], slots=1, budget_bytes=1 << 20)
    _add(srv, refs)
    srv.build()
    with pytest.raises(api.StormError, match="budget"):
        srv.submit(batches[2])
    srv.close()


def test_tight_budget_bounds_device_memory_and_every_batch_completes(world):
    """Under a budget far below what the batches would take at full speed, batches submitted
    together from several threads all complete (no out-of-memory): a pass that would need more
    than a slot's share of working memory maps its reads in halves, and a batch waits until the
    chains in flight leave room for its own.  Device memory in use, sampled while they run,
    never exceeds what the resident indexes took plus the budget (and a little for lazily loaded
    kernel code); every batch still gets the plain chain's results."""
    torch = pytest.importorskip("torch")
    _, refs, batches = world
    tbs = ((100 + ARGS["indels"] + 1) // 2 + 7) & ~7
    plain = [_plain_chain(refs, b, tbs) for b in batches]
    budget = 96 << 20
    torch.cuda.synchronize()
    free0, total = torch.cuda.mem_get_info()
    srv = api.Server(api.params(**ARGS), CHAIN, slots=3, budget_bytes=budget)
    _add(srv, refs)
    srv.build()
    _same(srv.poll(srv.submit(batches[0], tbs)), plain[0], "warm-up")
    free1, _ = torch.cuda.mem_get_info()
    resident = free0 - free1
    samples, stop = [], threading.Event()

    def sample():
        while not stop.is_set():
            samples.append(torch.cuda.mem_get_info()[0])
            stop.wait(0.002)
    th = threading.Thread(target=sample)
    th.start()
    rounds = 4  # every batch four times: a longer run to sample
    tickets = [None] * (rounds * len(batches))

    def go(i):
        tickets[i] = srv.submit(batches[i % len(batches)], tbs)
    ths = [threading.Thread(target=go, args=(i,)) for i in range(len(tickets))]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    outs = [srv.poll(t) for t in tickets]
    stop.set()
    th.join()
    srv.close()
    for i, out in enumerate(outs):
        _same(out, plain[i % len(batches)], ("tight", i))
    peak = max(free0 - f for f in samples) if samples else 0
    assert len(samples) >= 3
    assert peak <= resident + budget + (32 << 20), (peak >> 20, resident >> 20, budget >> 20)
