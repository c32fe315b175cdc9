"""stormgpu_align_noalloc, the alignment entry point that allocates nothing, against
stormgpu_align on the same inputs, through the C ABI.  Several calls in a row with different
reads, band widths, spaces and window counts (a larger call first), so that a result that
depended on what an earlier call left in the shared scratch array would show; then its size
limit and its window check, each followed by a call that must still agree."""
import numpy as np
import pytest

import ffi
from storm_b200 import api

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

PADB = 1024


def _mutate(rng, s, rate):
    s = s.copy()
    for i in range(len(s)):
        if rng.random() < rate:
            s[i] = (s[i] + rng.integers(1, 4)) & 3
    return s


def _case(rng, colour, I, L, G, nwin):
    g = rng.integers(0, 4, size=G).astype(np.uint8)
    m = np.zeros(G, np.uint8)
    for _ in range(3):
        a = int(rng.integers(0, G - 10))
        m[a:a + int(rng.integers(1, 8))] = 1
    src = int(rng.integers(0, G - L - 2 * I))
    read = _mutate(rng, g[src + I:src + I + L], 0.05)
    lv = rng.integers(0, 4, size=L).astype(np.uint8)
    hi = G - L - 2 * I
    wins = np.concatenate([[src], np.clip(src + rng.integers(-3, 4, size=nwin // 2), 0, hi),
                           rng.integers(0, hi + 1, size=nwin - 1 - nwin // 2)]).astype(np.int32)
    nb = (G + 3) // 4
    return dict(colour=colour, I=I, L=L, G=G, wins=wins,
                gp=ffi.pack2(g, PADB)[PADB:PADB + nb].copy(), mp=ffi.pack2(m, PADB, fill=0x55)[PADB:PADB + nb].copy(),
                rp=ffi.pack2(read), qp=ffi.pack2(lv))


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _noalloc(prm, c, wins=None):
    wins = c["wins"] if wins is None else wins
    n, L, I = len(wins), c["L"], c["I"]
    tbs = ((L + I + 1) // 2 + 7) & ~7
    d = {k: _dev(c[k]) for k in ("rp", "gp", "mp")}
    qaddr = _dev(c["qp"]) if c["qp"] is not None else None
    dw = _dev(wins)
    score = torch.empty(n, dtype=torch.int32, device="cuda")
    bound = torch.empty(n, dtype=torch.int32, device="cuda")
    best = torch.empty((n, 4), dtype=torch.int16, device="cuda")
    tbl = torch.empty(n, dtype=torch.int32, device="cuda")
    tb = torch.full((n, tbs), 0xAB, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    levels = qaddr.data_ptr() if qaddr is not None else 0
    api.align_noalloc(prm, d["rp"].data_ptr(), levels, L, d["gp"].data_ptr(), d["mp"].data_ptr(),
                      c["G"], dw.data_ptr(), n, score.data_ptr(), bound.data_ptr(), best.data_ptr(),
                      tbl.data_ptr(), tb.data_ptr(), tbs, torch.cuda.current_stream().cuda_stream)
    return score.cpu().numpy(), bound.cpu().numpy(), best.cpu().numpy(), tbl.cpu().numpy(), tb.cpu().numpy()


def _check_same(c):
    prm = api.params(colour=c["colour"], indels=c["I"])
    got = _noalloc(prm, c)
    exp = api.align(prm, c["rp"], c["qp"], c["L"], c["gp"], c["mp"], c["G"], c["wins"])
    for k in range(len(c["wins"])):
        ctx = (c["colour"], c["I"], c["L"], k, int(c["wins"][k]))
        assert got[0][k] == exp[0][k] and got[1][k] == exp[1][k], ctx
        assert tuple(got[2][k]) == tuple(exp[2][k]), ctx
        assert got[3][k] == exp[3][k], ctx
        nb = (int(exp[3][k]) + 1) // 2
        assert bytes(got[4][k, :nb]) == bytes(exp[4][k, :nb]), ctx
        assert not got[4][k, nb:].any(), ctx  # zero-filled after the traceback


def test_noalloc_matches_align_on_calls_in_a_row():
    rng = np.random.default_rng(2024)
    cases = [_case(rng, 1, 7, 100, 3000, 64),   # large first: fills more of the scratch
             _case(rng, 0, 3, 50, 1500, 9),
             _case(rng, 0, 15, 150, 4000, 33),
             _case(rng, 1, 0, 35, 800, 5)]
    for c in cases:
        _check_same(c)
    _check_same(cases[1])  # the same small call again, after a larger one


def test_noalloc_without_quality_levels():
    """levels = NULL (every level 3) in both calls, nucleotide and colour."""
    rng = np.random.default_rng(2025)
    for c in (_case(rng, 0, 7, 75, 2000, 17), _case(rng, 1, 3, 50, 1200, 11)):
        c["qp"] = None
        _check_same(c)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    rng = np.random.default_rng(7)
    L, I = 1000, 64
    c = _case(rng, 0, I, L, 4000, 240)  # 4 * 1000 * 9 * 240 bytes > 8 MiB
    prm = api.params(colour=0, indels=I)
    with pytest.raises(api.StormError, match="split the windows"):
        _noalloc(prm, c)
    small = dict(c, wins=c["wins"][:20])
    _check_same(small)


def test_noalloc_rejects_windows_outside_the_genome():
    rng = np.random.default_rng(8)
    c = _case(rng, 0, 3, 50, 1000, 6)
    prm = api.params(colour=0, indels=3)
    bad = c["wins"].copy()
    bad[2] = -5
    with pytest.raises(api.StormError, match="not inside"):
        _noalloc(prm, c, bad)
    bad[2] = c["G"] - c["L"] - 2 * c["I"] + 1
    with pytest.raises(api.StormError, match="not inside"):
        _noalloc(prm, c, bad)
    _check_same(c)
