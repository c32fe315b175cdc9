"""The wave schedule of the device contextual placement (storm_b200/csrc/genome_map_ctx.cu),
restated in Python and checked on the CPU against the host restatement of the reference's
one-by-one placement (storm_host.c sh_genome_map_contextual, pinned to the reference by the
command-line tests, genome_map.c:233-531): reads placed in waves -- each wave, the pending reads
that hold the earliest rank on every position of their candidate spans, in any order within the
wave -- give the placements of the sequential order, on records built to pile many reads with
several candidates each on a few kilobases."""
import ctypes as C

import numpy as np
import pytest

from storm_b200 import api, build, host, synth

MIN_SCORE = api.MIN_SCORE
NO_CODE = 4


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def _get6(c, s):
    return (c >> (6 * s)) & 0x3F


def _inc6(c, s):
    v = (_get6(c, s) + 1) & 0x3F
    return (c & ~(0x3F << (6 * s)) & 0xFFFFFFFF) | (v << (6 * s))


def _pair_type(code, colour):
    if (code & 0xC) == 0x4:
        return 0x4
    if colour and (code & 0xC) == 0x8:
        return 0x8
    if (code & 0xC) == 0xC:
        return 0xC
    return code


class WaveModel:
    def __init__(self, refs, hits, ops, mapped, colour, indels, match, mismatch):
        self.refs, self.hits, self.ops, self.mapped = refs, hits, ops, mapped
        self.colour, self.I, self.match, self.mismatch = colour, indels, match, mismatch
        self.base = np.concatenate([[0], np.cumsum([len(r) + 1 for r in refs])])[:-1]
        self.state = {}  # global position -> [created, aligned, inserted counters]

    def cands(self, r):
        k = 0
        while k < 4 and self.hits[r][k] is not None:
            k += 1
        return k

    def span(self, r, k):
        ref, start = self.hits[r][k][1], self.hits[r][k][2]
        a = int(self.base[ref]) + start
        return a, min(a + len(self.ops[r][k]), int(self.base[ref]) + len(self.refs[ref]))

    def positions(self, r):
        for k in range(self.cands(r)):
            a, b = self.span(r, k)
            yield from range(a, b + 1)

    def consensus(self, gp, offset, ref_code):
        st = self.state.get(gp)
        if st is None or not st[0] or offset >= self.I:
            return ref_code
        cnt = st[1] if offset < 0 else st[2][offset]
        best = ref_code
        for s in range(NO_CODE + 1):
            if _get6(cnt, s) > _get6(cnt, best):
                best = s
        return NO_CODE if _get6(cnt, best) == 0 else best

    def update(self, gp, offset, code):
        st = self.state.setdefault(gp, [False, 0, [0] * max(self.I, 1)])
        st[0] = True
        if offset >= 0:
            if offset < self.I:
                st[2][offset] = _inc6(st[2][offset], code)
        else:
            st[1] = _inc6(st[1], code)

    def adjusted(self, r, k):
        ref, start = self.hits[r][k][1], self.hits[r][k][2]
        a, b = self.span(r, k)
        score, indel, pos, gp = 0, 0, start, a
        for cell in self.ops[r][k]:
            if gp > b:
                break
            t = _pair_type(cell, self.colour)
            if t == 0x3:
                rc = int(self.refs[ref][pos])
                score += self.match if rc == self.consensus(gp, -1, rc) else self.mismatch
                pos, gp, indel = pos + 1, gp + 1, 0
            elif t == 0x1:
                score += self.match if self.consensus(gp, -1, NO_CODE) == NO_CODE else self.mismatch
                pos, gp, indel = pos + 1, gp + 1, 0
            elif t in (0x4, 0x8):
                c = cell & 3
                score += self.match if c == self.consensus(gp, -1, c) else self.mismatch
                pos, gp, indel = pos + 1, gp + 1, 0
            elif t == 0xC:
                c = cell & 3
                score += self.match if c == self.consensus(gp, indel, c) else self.mismatch
                indel += 1
        return score

    def place(self, r, uniqueness, threshold):
        nk = self.cands(r)
        adj = [MIN_SCORE] * 4
        best_rank, best = -1, MIN_SCORE
        for k in range(nk):
            adj[k] = self.adjusted(r, k)
            if adj[k] > best:
                best, best_rank = adj[k], k
        if best_rank < 0 or (uniqueness and not (adj[0] - adj[1] > threshold)):
            return -1
        ref, start = self.hits[r][best_rank][1], self.hits[r][best_rank][2]
        a, b = self.span(r, best_rank)
        self.state.setdefault(a, [False, 0, [0] * max(self.I, 1)])[0] = True
        pos, gp, ins = start, a, -1
        for cell in self.ops[r][best_rank]:
            if gp > b:
                break
            t = _pair_type(cell, self.colour)
            if t == 0xC:
                ins += 1
                self.update(gp, ins, cell & 3)
            elif t == 0x3:
                ins = -1
                self.update(gp, -1, int(self.refs[ref][pos]))
            elif t in (0x4, 0x8):
                ins = -1
                self.update(gp, -1, cell & 3)
            elif t == 0x1:
                ins = -1
                self.update(gp, -1, NO_CODE)
            for p in range(ins + 1, self.I):
                self.update(gp, p, NO_CODE)
            if ins < 0:
                pos, gp = pos + 1, gp + 1
        return best_rank

    def run(self, uniqueness, threshold, rng):
        idx = [r for r in range(len(self.hits)) if self.mapped[r]]
        order = sorted(idx, key=lambda r: -(self.hits[r][0][0] & 0xFFFFFFFF))  # stable: read order in ties
        placed = {}
        pending = list(range(len(order)))
        waves = 0
        while pending:
            minrank = {}
            for j in pending:
                for p in self.positions(order[j]):
                    minrank[p] = min(minrank.get(p, len(order)), j)
            ready = [j for j in pending if all(minrank[p] == j for p in self.positions(order[j]))]
            assert ready and ready[0] == pending[0]
            for j in rng.permutation(ready):
                placed[int(j)] = self.place(order[int(j)], uniqueness, threshold)
            done = set(ready)
            pending = [j for j in pending if j not in done]
            waves += 1
        out = [(int(self.base[self.hits[order[j]][k][1]]) + self.hits[order[j]][k][2], j, order[j], k)
               for j, k in placed.items() if k >= 0]
        out.sort()
        return [(r, k) for _, _, r, k in out], waves


def _records(rng, refs, n, colour, indels):
    hits, ops, mapped = [], [], []
    # the operations a traceback holds (alignment.h:59-78): match, code mismatch, read insertion (at
    # most `indels` in a row), read deletion, colour-base mismatch in colour space
    kinds = [3] * 14 + [4, 5, 6, 7] + [12, 13, 14, 15] + [1, 1] + ([8, 9, 10, 11] if colour else [])
    for _ in range(n):
        row, orow = [None] * 4, [None] * 4
        m = rng.random() < 0.9
        for k in range(int(rng.integers(1, 5)) if m else 0):
            ref = int(rng.integers(0, len(refs)))
            length = int(rng.integers(20, 60))
            cells, run = [], 0
            for _ in range(length):
                c = int(rng.choice(kinds))
                if (c & 0xC) == 0xC:
                    if run >= indels:
                        c = 3
                    else:
                        run += 1
                if (c & 0xC) != 0xC:
                    run = 0
                cells.append(c)
            start = int(rng.integers(0, len(refs[ref]) - length - 1))
            row[k] = (int(rng.integers(-60, 260)), ref, start)
            orow[k] = cells
        hits.append(row)
        ops.append(orow)
        mapped.append(1 if m and row[0] is not None else 0)
    return hits, ops, mapped


def _host_placement(refs_s, hits, ops, mapped, colour, indels, match, mismatch, uniqueness, threshold):
    n = len(hits)
    tbs = 40
    h = np.zeros(n * 4, api.HIT_DTYPE)
    h["ref_start"] = -1
    h["ref_id"] = -1
    h["score"] = MIN_SCORE
    tb = np.zeros((n * 4, tbs), np.uint8)
    for r in range(n):
        for k in range(4):
            if hits[r][k] is None:
                continue
            s, ref, start = hits[r][k]
            i = r * 4 + k
            h["score"][i], h["ref_id"][i], h["ref_start"][i] = s, ref, start
            h["tb_len"][i], h["sense"][i] = len(ops[r][k]), 1
            for i, c in enumerate(ops[r][k]):
                tb[r * 4 + k, i >> 1] |= c << (0 if i & 1 else 4)
    mp = np.array(mapped, np.uint8)
    res = api.Results(h.ctypes.data, tb.ctypes.data, tbs, mp.ctypes.data)
    L = host.hostlib()
    L.sh_genome_map_contextual.argtypes = [C.POINTER(host.ShRefs), C.POINTER(api.Results), C.c_int64, C.c_int,
                                           C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                           C.POINTER(C.c_int64)]
    out = np.zeros((max(n, 1), 2), np.int32)
    npl = C.c_int64(0)
    assert L.sh_genome_map_contextual(C.byref(refs_s), C.byref(res), n, colour, indels, match, mismatch, uniqueness,
                                      threshold, out.ctypes.data, C.byref(npl)) == 0
    return [(int(a), int(b)) for a, b in out[:npl.value]]


@pytest.mark.parametrize("colour,indels,uniqueness,threshold,seed", [
    (0, 3, 0, 0, 1), (0, 7, 1, 5, 2), (1, 5, 0, 0, 3), (1, 2, 1, 3, 4), (0, 1, 0, 0, 5)])
def test_waves_give_the_sequential_placement(tmp_path, colour, indels, uniqueness, threshold, seed):
    genome = synth.make_genome([3000, 1800], 40 + seed, 0.45, 0.3)
    synth.write_fasta(str(tmp_path / "ref.fa"), genome)
    ref = host.Reference(str(tmp_path / "ref.fa"), colour)
    s = ref._s
    refs = []
    for k in range(s.n):
        size = int(s.sizes[k])
        raw = np.frombuffer(C.string_at(s.codes[k], (size + 3) // 4), np.uint8)
        refs.append(((raw[np.arange(size) >> 2] >> ((np.arange(size) & 3) * 2)) & 3).astype(np.int64))
    rng = np.random.default_rng(seed)
    hits, ops, mapped = _records(rng, refs, 500, colour, indels)
    want = _host_placement(s, hits, ops, mapped, colour, indels, 5, -4, uniqueness, threshold)
    for trial in range(2):
        model = WaveModel(refs, hits, ops, mapped, colour, indels, 5, -4)
        got, waves = model.run(uniqueness, threshold, np.random.default_rng(seed * 10 + trial))
        assert got == want, (trial, waves)
    assert waves > 10 and len(want) > 100
    assert any(k > 0 for _, k in want)
