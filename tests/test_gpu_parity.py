"""GPU parity: every CUDA kernel against the oracle on seeded inputs, through the C ABI.

Bar: bit-exact (integer work).  The oracle itself is pinned to the reference by
tests/test_oracle_pin.py and tests/test_e2e_cpu.py."""
import ctypes as C

import numpy as np
import pytest

import ffi
from storm_b200 import api, build

pytestmark = pytest.mark.gpu

PADB = 128


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()
    if not api.device_available():
        pytest.fail("no CUDA device: GPU tests need a B200")


def _mutate(rng, s, rate):
    s = s.copy()
    m = rng.random(len(s)) < rate
    s[m] = (s[m] + rng.integers(1, 4, size=int(m.sum()))) % 4
    return s


@pytest.mark.parametrize("W", [2, 4, 8, 16])
def test_filter_kernel_vs_oracle(W):
    rng = np.random.default_rng(200 + W)
    orc = ffi.oracle()
    G = 5000
    g = rng.integers(0, 4, size=G).astype(np.uint8)
    gp = ffi.pack2(g, PADB)
    base = gp.ctypes.data + PADB
    total = passed = 0
    for trial in range(40):
        L = int(rng.choice([3, 12, 35, 49, 50, 75, 100, 150, 151, 250]))
        match = int(rng.choice([5, 5, 3, 9, 300]))
        mism, go, ge = int(rng.choice([4, 3])), int(rng.choice([9, 7])), int(rng.choice([4, 2]))
        thr = int(rng.choice([40, 80, 100, 150, 254, 400]))
        src = int(rng.integers(0, G - L - 40))
        read = _mutate(rng, g[src:src + L], rng.choice([0.0, 0.05, 0.2, 0.75]))
        rp = np.concatenate([ffi.pack2(read), np.zeros(64, np.uint8)])
        n = 96
        pos = np.concatenate([src - rng.integers(0, 2 * W, size=n // 3),
                              rng.integers(-L - 8, G + 8, size=n - n // 3)]).astype(np.int32)
        got = api.sw_filter(W, L, match, mism, go, ge, thr, gp[PADB:PADB + (G + 3) // 4], G, pos, rp)
        for k in range(n):
            exp = orc.or_sw_filter(W, L, match, mism, go, ge, thr, C.c_void_p(base), int(pos[k]), rp.ctypes.data)
            assert got[k] == exp, (trial, k, W, L, match, thr, int(pos[k]))
        total += n
        passed += int(got.sum())
    assert 0 < passed < total


@pytest.mark.parametrize("colour", [0, 1])
def test_align_kernel_vs_oracle(colour):
    rng = np.random.default_rng(31 + colour)
    orc = ffi.oracle()
    G = 2000
    for trial in range(60):
        I = int(rng.choice([0, 1, 2, 3, 5, 7, 10, 15, 20, 31]))
        L = int(rng.choice([8, 20, 35, 49, 50, 75, 100, 150, 300]))
        match, mism = int(rng.choice([5, 3])), int(rng.choice([-4, -3, -6]))
        go, ge = int(rng.choice([-9, -7])), int(rng.choice([-4, -2]))
        g = rng.integers(0, 4, size=G).astype(np.uint8)
        m = np.zeros(G, np.uint8)
        for _ in range(int(rng.integers(0, 3))):
            a = int(rng.integers(0, G - 10))
            m[a:a + int(rng.integers(1, 8))] = 1
        gp = ffi.pack2(g, PADB)
        mp = ffi.pack2(m, PADB, fill=0x55)
        src = int(rng.integers(0, G - L - 2 * I))
        read = _mutate(rng, g[src + I:src + I + L], rng.choice([0.0, 0.03, 0.1, 0.3]))
        lv = rng.integers(0, 4, size=L).astype(np.uint8)
        rp = ffi.pack2(read)
        qp = ffi.pack2(lv)
        use_q = rng.random() < 0.8
        wins = np.concatenate([[src], src + rng.integers(-3, 4, size=3),
                               rng.integers(-L - 2 * I, G, size=4)]).astype(np.int32)
        prm = api.params(colour=colour, match=match, mismatch=mism, gap_open=go, gap_extend=ge, indels=I)
        score, bound, best, tbl, tb = api.align(prm, rp, qp if use_q else None, L, gp[PADB:PADB + (G + 3) // 4],
                                                mp[PADB:PADB + (G + 3) // 4], G, wins)
        p = ffi.make_params(colour=colour, match=match, mismatch=mism, gap_open=go, gap_extend=ge, indels=I)
        for k, w in enumerate(wins):
            o = ffi.OrAlignOut()
            orc.or_align(C.byref(p), C.c_void_p(rp.ctypes.data), C.c_void_p(qp.ctypes.data if use_q else 0),
                         L, C.c_void_p(gp.ctypes.data + PADB), C.c_void_p(mp.ctypes.data + PADB),
                         C.c_int64(int(w)), C.byref(o))
            ctx = (trial, k, colour, I, L, int(w))
            assert score[k] == o.score and bound[k] == o.bound, ctx
            assert tuple(best[k]) == (o.best_i, o.best_j, o.best_i0, o.best_j0), ctx
            assert tbl[k] == o.tb_len, ctx
            nb = (o.tb_len + 1) // 2
            assert bytes(tb[k, :nb]) == bytes(o.tb)[:nb], ctx


def test_index_kernel_vs_oracle():
    rng = np.random.default_rng(17)
    orc = ffi.oracle()
    for trial, (N, seed, l) in enumerate([(100000, "####--#-#--##--####", 100), (50000, "#####-##-###", 3),
                                          (30000, "##-##-###-###", 0), (20000, "###-#-###", 1),
                                          (5000, "######", 100), (300, "####-##", 2)]):
        g = rng.integers(0, 4, size=N).astype(np.uint8)
        for _ in range(30 if N > 1000 else 0):
            a, b = rng.integers(0, N - 300, size=2)
            g[b:b + 200] = g[a:a + 200]
        regs = [(N // 3, N // 3 + 50), (N // 2, N // 2 + 3), (N - 7, N)]
        gp = ffi.pack2(g, PADB)
        first, mp = api.index_one(seed, l, gp[PADB:PADB + (N + 3) // 4], N, regs)
        sb = C.create_string_buffer(16 * 2048)
        assert orc.or_parse_seeds(seed.encode(), sb, 16) == 1
        f2 = np.zeros_like(first)
        m2 = np.zeros(N + 64, np.int32)
        rs = np.array([a for a, _ in regs], np.int32)
        re_ = np.array([b for _, b in regs], np.int32)
        n2 = orc.or_index_build(sb, l, C.c_void_p(gp.ctypes.data + PADB), C.c_int64(N), rs.ctypes.data,
                                re_.ctypes.data, len(regs), f2.ctypes.data, m2.ctypes.data, C.c_int64(len(m2)))
        assert n2 == len(mp), trial
        assert np.array_equal(first, f2), trial
        assert np.array_equal(mp, m2[:n2]), trial


def _reads_arrays(seqs, quals, colour_first_levels=None):
    n = len(seqs)
    maxl = max(len(s) for s in seqs)
    stride = ((maxl + 3) // 4 + 7) & ~7
    codes = np.zeros((n, stride), np.uint8)
    levels = np.zeros((n, stride), np.uint8)
    for i, (s, q) in enumerate(zip(seqs, quals)):
        p = ffi.pack2(s)
        codes[i, :len(p)] = p
        lv = np.searchsorted(np.array([2, 7, 10]), np.asarray(q), side="left").astype(np.uint8)
        lp = ffi.pack2(lv)
        levels[i, :len(lp)] = lp
    return codes, levels, np.array([len(s) for s in seqs], np.int16)


def _masked_runs(n, rng, frac=0.004):
    """Masked runs (start, end) of 1-30 codes covering about `frac` of n codes, and the 0/1 mask."""
    m = np.zeros(n, np.uint8)
    runs = []
    pos = int(rng.integers(0, 400))
    while True:
        pos += int(rng.integers(1, int(30 / frac)))
        if pos >= n - 40:
            break
        ln = int(rng.integers(1, 31))
        m[pos:pos + ln] = 1
        runs.append((pos, pos + ln))
        pos += ln
    return runs, m


@pytest.mark.parametrize("colour,indels,seeds,masked,min_score", [
    (0, 3, "####--#-#--##--####;#####--###-#-###;###-##-#######", False, 100),
    (0, 15, "##-##-###-###;###--#-#--#--####", False, 100),
    (1, 7, "####-##-#-####;###-#--##-##--###;####-#---#----#--####", False, 110),
    # masked reference runs (alignment rows with masked cells), every constant band width
    (0, 7, "####--#-#--##--####;#####--###-#-###;###-##-#######", True, 100),
    (0, 15, "##-##-###-###;###--#-#--#--####", True, 60),
    (0, 20, "##-##-###-###;###--#-#--#--####", True, 100),
])
def test_map_api_vs_oracle(colour, indels, seeds, masked, min_score):
    from storm_b200 import synth
    genome = synth.make_genome([40000, 15000], 21, gc=0.45, repeat_frac=0.2)
    rng = np.random.default_rng(77)
    masks = [_masked_runs(len(s), rng) if masked else ([], np.zeros(len(s), np.uint8)) for _, s in genome]
    if colour:
        pr, cols, q = synth.simulate_colour_reads(genome, 1500, 40, 22)
        seqs = [c for c in cols]
        quals = [qq for qq in q]
        # colour-space reference: colours of consecutive bases
        refs = [(n, (s[1:] ^ s[:-1]).astype(np.uint8)) for n, s in genome]
    else:
        seqs, quals = synth.simulate_nucleotide_reads(genome, 2000, [35, 50, 75, 100, 150], 23)
        refs = genome
    codes, levels, lengths = _reads_arrays(seqs, quals)
    first_levels = np.full(len(seqs), 2, np.uint8) if colour else None
    prm = api.params(colour=colour, indels=indels, min_score=min_score, min_score_filter=95)
    m = api.Mapper(prm, seeds)
    packed = []
    for (name, s), (runs, mask) in zip(refs, masks):
        cp = ffi.pack2(s, PADB)
        mk = ffi.pack2(mask[:len(s)], PADB, fill=0x55)
        packed.append((cp, mk, len(s), runs))
        m.add_reference(cp[PADB:], mk[PADB:], len(s), regions=runs)
    m.build_index()
    batch = api.ReadBatch(codes, lengths, levels, first_levels)
    res = m.map(batch)
    st = m.stats()
    m.close()
    # oracle
    orc = ffi.oracle()
    R = (ffi.OrRef * len(packed))()
    keep = []
    for k, (cp, mk, n, runs) in enumerate(packed):
        rs = np.array([a for a, _ in runs] or [0], np.int32)
        re = np.array([b for _, b in runs] or [0], np.int32)
        keep += [rs, re]
        R[k] = ffi.OrRef(cp.ctypes.data + PADB, mk.ctypes.data + PADB, n, rs.ctypes.data, re.ctypes.data, len(runs))
    rd = ffi.ReadsT(len(seqs), codes.ctypes.data, codes.shape[1], levels.ctypes.data, levels.shape[1],
                    lengths.ctypes.data, first_levels.ctypes.data if colour else None)
    hits = np.zeros(len(seqs) * 4, dtype=api.HIT_DTYPE)
    tb = np.zeros((len(seqs) * 4, res.tb_stride), np.uint8)
    mapped = np.zeros(len(seqs), np.uint8)
    out = ffi.ResultsT(hits.ctypes.data, tb.ctypes.data, res.tb_stride, mapped.ctypes.data)
    p = ffi.make_params(colour=colour, indels=indels, min_score=min_score, min_score_filter=95)
    cnt = np.zeros(3, np.int64)
    assert orc.or_map(C.byref(p), seeds.encode(), R, len(packed), C.byref(rd), C.byref(out), cnt.ctypes.data) == 0
    assert np.array_equal(res.mapped, mapped)
    assert np.array_equal(res.hits, hits)
    for k in range(len(hits)):
        nb = (hits[k]["tb_len"] + 1) // 2
        assert bytes(res.tb[k, :nb]) == bytes(tb[k, :nb]), k
    assert mapped.sum() > len(seqs) // 4
    assert st["filter_passed"] == cnt[1]


def test_map_is_invariant_to_read_order_in_a_mixed_length_batch():
    """A batch of reads of several lengths is gathered grouped by length (a device sort of the
    read indices); the results of a read must not depend on where it sits in the batch."""
    from storm_b200 import synth
    genome = synth.make_genome([60000], 31, gc=0.42, repeat_frac=0.25)
    seqs, quals = synth.simulate_nucleotide_reads(genome, 3000, [35, 50, 75, 100, 150], 31)
    codes, levels, lengths = _reads_arrays(seqs, quals)
    prm = api.params(indels=15, min_score=100, min_score_filter=95)
    m = api.Mapper(prm, "##-##-###-###;###--#-#--#--####")
    for _, s in genome:
        cp = ffi.pack2(s, PADB)
        mk = ffi.pack2(np.zeros(len(s), np.uint8), PADB, fill=0x55)
        m.add_reference(cp[PADB:], mk[PADB:], len(s))
    m.build_index()
    tbs = ((150 + 15 + 1) // 2 + 7) & ~7
    base = m.map(api.ReadBatch(codes, lengths, levels), tbs)
    perm = np.random.default_rng(5).permutation(len(seqs))
    shuf = m.map(api.ReadBatch(codes[perm], lengths[perm], levels[perm]), tbs)
    order = np.argsort(lengths, kind="stable")
    srt = m.map(api.ReadBatch(codes[order], lengths[order], levels[order]), tbs)
    m.close()
    assert base.mapped.sum() > len(seqs) // 4
    for got, p in ((shuf, perm), (srt, order)):
        assert np.array_equal(got.mapped, base.mapped[p])
        h4 = (4 * p[:, None] + np.arange(4)).ravel()
        assert got.hits.tobytes() == base.hits[h4].tobytes()
        live = np.nonzero(got.hits["ref_id"] >= 0)[0]
        for k in live:
            nb = (int(got.hits["tb_len"][k]) + 1) // 2
            assert bytes(got.tb[k, :nb]) == bytes(base.tb[h4[k], :nb]), k


def test_map_results_do_not_depend_on_the_launch_tuning():
    """The launch parameters (hit bucket, reads per steal, filter tile rows, alignment run per
    steal) and the autotuner that picks them change no result."""
    from storm_b200 import synth
    genome = synth.make_genome([80000], 41, gc=0.42, repeat_frac=0.4)
    seqs, quals = synth.simulate_nucleotide_reads(genome, 2500, [35, 75, 150], 43)
    codes, levels, lengths = _reads_arrays(seqs, quals)
    prm = api.params(indels=15, min_score=100, min_score_filter=95)
    m = api.Mapper(prm, "##-##-###-###;###--#-#--#--####")
    for _, s in genome:
        cp = ffi.pack2(s, PADB)
        mk = ffi.pack2(np.zeros(len(s), np.uint8), PADB, fill=0x55)
        m.add_reference(cp[PADB:], mk[PADB:], len(s))
    m.build_index()
    batch = api.ReadBatch(codes, lengths, levels)
    tbs = ((150 + 15 + 1) // 2 + 7) & ~7
    assert m.tuning() == {"gather_warp_cap": 768, "gather_reads_per_steal": 4, "filter_rows": 8, "align_steal": 32,
                          "filter_cursor": 0, "align_rounds": 4}
    base = m.map(batch, tbs)
    st = m.stats()
    assert base.mapped.sum() > len(seqs) // 4
    settings = [dict(gather_warp_cap=256, gather_reads_per_steal=1, filter_rows=1, align_steal=1024, filter_cursor=1,
                     align_rounds=1),
                dict(gather_warp_cap=1536, gather_reads_per_steal=64, filter_rows=64, align_steal=32, filter_cursor=0,
                     align_rounds=6),
                dict(gather_warp_cap=1000, gather_reads_per_steal=3, filter_rows=5, align_steal=96, filter_cursor=1,
                     align_rounds=2)]
    for kw in settings:
        m.set_tuning(**kw)
        got = m.map(batch, tbs)
        assert m.stats()["candidates"] == st["candidates"], kw
        assert np.array_equal(got.mapped, base.mapped), kw
        assert got.hits.tobytes() == base.hits.tobytes(), kw
        assert got.tb.tobytes() == base.tb.tobytes(), kw
    with pytest.raises(api.StormError, match="out of range"):
        m.set_tuning(align_steal=48)
    picked = m.autotune(batch, sample=1500)
    assert m.tuning() == picked
    got = m.map(batch, tbs)
    assert got.hits.tobytes() == base.hits.tobytes() and got.tb.tobytes() == base.tb.tobytes()
    m.close()


def _same_results(got, base):
    assert np.array_equal(got.mapped, base.mapped)
    assert got.hits.tobytes() == base.hits.tobytes()
    assert got.tb.tobytes() == base.tb.tobytes()


def _stage_sums(st):
    return {k: st[k] for k in ("candidates", "filter_passed", "aligned", "seed_lookups", "hit_positions",
                               "filter_cells", "filter_band_cells", "align_cells", "passes")}


def test_graph_passes_give_the_host_synced_results():
    """From a context's second mapping call on, every strand pass of a call runs inside one CUDA
    graph, its lists sized from the densest pass seen so far and every launch taking its list
    size from device memory.  Results and stage counters must be those of the passes run as
    separate launches with the host reading each size, for one alignment round and for several."""
    from storm_b200 import synth
    genome = synth.make_genome([80000], 61, gc=0.42, repeat_frac=0.4)
    seqs, quals = synth.simulate_nucleotide_reads(genome, 2500, [35, 75, 150], 63)
    codes, levels, lengths = _reads_arrays(seqs, quals)
    prm = api.params(indels=15, min_score=100, min_score_filter=95)
    batch = api.ReadBatch(codes, lengths, levels)
    tbs = ((150 + 15 + 1) // 2 + 7) & ~7

    def mapper(graphs):
        m = api.Mapper(prm, "##-##-###-###;###--#-#--#--####")
        for _, s in genome:
            cp = ffi.pack2(s, PADB)
            mk = ffi.pack2(np.zeros(len(s), np.uint8), PADB, fill=0x55)
            m.add_reference(cp[PADB:], mk[PADB:], len(s))
        m.build_index()
        m.set_graphs(graphs)
        return m

    plain, g = mapper(False), mapper(True)
    for rounds in (4, 1, 3):
        plain.set_tuning(align_rounds=rounds)
        g.set_tuning(align_rounds=rounds)
        base = plain.map(batch, tbs)
        sb = plain.stats()
        assert sb["graph_passes"] == 0 and sb["passes"] == 2
        for _ in range(2):
            got = g.map(batch, tbs)
            sg = g.stats()
            _same_results(got, base)
            assert _stage_sums(sg) == _stage_sums(sb)
        assert sg["graph_passes"] == sg["passes"] == 2, sg
        assert sg["ms_filter"] > 0 and sg["ms_gather"] > 0 and sg["ms_total"] > 0, sg
    plain.close()
    g.close()
    assert base.mapped.sum() > len(seqs) // 4


def test_graph_call_whose_lists_outgrow_their_sizes_runs_again():
    """A graph call sizes its lists from the last call: after reads from unique sequence, reads of
    a 600-copy tandem repeat (a 150-bp read gathers about 200,000 index positions on its strand,
    and has hundreds of candidates and passing candidates) outgrow the passing-candidate list and
    the slices of the gather for reads with the most positions.  That call must run again as
    separate launches and give the results of a context without graphs; the next call of the
    same batch then fits its graph."""
    from storm_b200 import synth
    rng = np.random.default_rng(91)
    unit = synth.random_bases(rng, 1000, 0.45)
    flank = synth.random_bases(rng, 40000, 0.45)
    g_ = np.concatenate([flank] + [_mutate(rng, unit, 0.02) for _ in range(600)] +
                        [synth.random_bases(rng, 20000, 0.45)])
    seqs, quals = synth.simulate_nucleotide_reads([("chr1", g_[20000:])], 400, [50, 150], 92)
    codes, levels, lengths = _reads_arrays(seqs, quals)
    useq, uqual = synth.simulate_nucleotide_reads([("flank", flank)], 300, [150], 93)
    ucodes, ulevels, ulengths = _reads_arrays(useq, uqual)
    prm = api.params(indels=15, min_score=100, min_score_filter=100)
    tbs = ((150 + 15 + 1) // 2 + 7) & ~7
    batch = api.ReadBatch(codes, lengths, levels)
    unique = api.ReadBatch(ucodes, ulengths, ulevels)

    def mapper(graphs):
        m = api.Mapper(prm, "##-##-###-###;###--#-#--#--####;####--#--#---#---###")
        cp = ffi.pack2(g_, PADB)
        mk = ffi.pack2(np.zeros(len(g_), np.uint8), PADB, fill=0x55)
        m.add_reference(cp[PADB:], mk[PADB:], len(g_))
        m.build_index()
        m.set_graphs(graphs)
        return m

    plain, g = mapper(False), mapper(True)
    ubase = plain.map(unique, tbs)
    base = plain.map(batch, tbs)
    sb = plain.stats()
    assert sb["hit_positions"] / len(seqs) > 50000, sb
    assert sb["candidates"] > 100000 and sb["filter_passed"] > 20000, sb
    _same_results(g.map(unique, tbs), ubase)
    assert g.stats()["graph_passes"] == 0  # no density yet: separate launches
    _same_results(g.map(unique, tbs), ubase)
    assert g.stats()["graph_passes"] == 2
    _same_results(g.map(batch, tbs), base)  # outgrows the sizes of the unique reads
    st = g.stats()
    assert st["graph_passes"] == 0 and _stage_sums(st) == _stage_sums(sb), st
    _same_results(g.map(batch, tbs), base)
    st = g.stats()
    assert st["graph_passes"] == 2 and _stage_sums(st) == _stage_sums(sb), st
    plain.close()
    g.close()
    assert base.mapped.sum() > len(seqs) // 2


def test_large_host_batch_gives_the_small_batch_results():
    """A host-buffer batch of a million reads (3,000 distinct reads repeated): every read's
    result must be the one it gets in a batch of its own 3,000."""
    from storm_b200 import synth
    genome = synth.make_genome([50000], 51, gc=0.45, repeat_frac=0.2)
    seqs, quals = synth.simulate_nucleotide_reads(genome, 3000, [50], 53)
    codes, levels, lengths = _reads_arrays(seqs, quals)
    prm = api.params(indels=3, min_score=100, min_score_filter=95)
    m = api.Mapper(prm, "####--#-#--##--####;#####--###-#-###;###-##-#######")
    for _, s in genome:
        cp = ffi.pack2(s, PADB)
        mk = ffi.pack2(np.zeros(len(s), np.uint8), PADB, fill=0x55)
        m.add_reference(cp[PADB:], mk[PADB:], len(s))
    m.build_index()
    small = m.map(api.ReadBatch(codes, lengths, levels))
    st_small = m.stats()
    rep = 350  # 1,050,000 reads
    big = m.map(api.ReadBatch(np.tile(codes, (rep, 1)), np.tile(lengths, rep), np.tile(levels, (rep, 1))))
    st_big = m.stats()
    m.close()
    assert small.mapped.sum() > 1000
    assert st_big["candidates"] == rep * st_small["candidates"]
    assert np.array_equal(big.mapped, np.tile(small.mapped, rep))
    assert big.hits.tobytes() == np.tile(small.hits, rep).tobytes()
    assert big.tb.tobytes() == np.tile(small.tb, (rep, 1)).tobytes()


def _oracle_map(packed, seeds, codes, levels, lengths, tbs, indels, min_score, min_score_filter):
    orc = ffi.oracle()
    R = (ffi.OrRef * len(packed))()
    keep = []
    for k, (cp, mk, n, runs) in enumerate(packed):
        rs = np.array([a for a, _ in runs] or [0], np.int32)
        re = np.array([b for _, b in runs] or [0], np.int32)
        keep += [rs, re]
        R[k] = ffi.OrRef(cp.ctypes.data + PADB, mk.ctypes.data + PADB, n, rs.ctypes.data, re.ctypes.data, len(runs))
    n = len(lengths)
    rd = ffi.ReadsT(n, codes.ctypes.data, codes.shape[1], levels.ctypes.data, levels.shape[1], lengths.ctypes.data,
                    None)
    hits = np.zeros(n * 4, dtype=api.HIT_DTYPE)
    tb = np.zeros((n * 4, tbs), np.uint8)
    mapped = np.zeros(n, np.uint8)
    out = ffi.ResultsT(hits.ctypes.data, tb.ctypes.data, tbs, mapped.ctypes.data)
    p = ffi.make_params(colour=0, indels=indels, min_score=min_score, min_score_filter=min_score_filter)
    assert orc.or_map(C.byref(p), seeds.encode(), R, len(packed), C.byref(rd), C.byref(out), None) == 0
    return hits, tb, mapped


def test_map_of_tandem_repeats_vs_oracle():
    """Reads from 300 mutated copies of one 1,000-bp unit: every seed key of such a read occurs
    about 250 times, so a 150-bp read-strand gathers about 100,000 index positions -- the
    block-per-read gather and its large-slice second launch -- and every read has hundreds of
    passing candidates, aligned in several rounds whose later ones stop early."""
    from storm_b200 import synth
    rng = np.random.default_rng(77)
    unit = synth.random_bases(rng, 1000, 0.45)
    copies = [_mutate(rng, unit, 0.02) for _ in range(300)]
    g = np.concatenate([synth.random_bases(rng, 20000, 0.45)] + copies + [synth.random_bases(rng, 20000, 0.45)])
    genome = [("chr1", g)]
    seqs, quals = synth.simulate_nucleotide_reads(genome, 600, [50, 150], 78)
    codes, levels, lengths = _reads_arrays(seqs, quals)
    seeds = "##-##-###-###;###--#-#--#--####;####--#--#---#---###"
    prm = api.params(indels=15, min_score=100, min_score_filter=100)
    m = api.Mapper(prm, seeds)
    cp = ffi.pack2(g, PADB)
    mk = ffi.pack2(np.zeros(len(g), np.uint8), PADB, fill=0x55)
    m.add_reference(cp[PADB:], mk[PADB:], len(g))
    m.build_index()
    tbs = ((150 + 15 + 1) // 2 + 7) & ~7
    batch = api.ReadBatch(codes, lengths, levels)
    results = []
    for rounds in (1, 4, 6):
        m.set_tuning(align_rounds=rounds)
        results.append(m.map(batch, tbs))
        st = m.stats()
        assert st["hit_positions"] / len(seqs) > 20000, st  # the strand a read came from gathers ~50,000
    m.close()
    hits, tb, mapped = _oracle_map([(cp, mk, len(g), [])], seeds, codes, levels, lengths, tbs, 15, 100, 100)
    assert mapped.sum() > len(seqs) // 2
    for res in results:
        assert np.array_equal(res.mapped, mapped)
        assert res.hits.tobytes() == hits.tobytes()
        for k in np.nonzero(hits["ref_id"] >= 0)[0]:
            nb = (int(hits["tb_len"][k]) + 1) // 2
            assert bytes(res.tb[k, :nb]) == bytes(tb[k, :nb]), k
