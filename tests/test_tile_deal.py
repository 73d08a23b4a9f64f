"""The hot phases' host-side tiling (``noaidi_b200/csrc/prima_tiles.cpp``),
built alone with the host compiler and checked on the CPU.

* the tile table covers every row once, tiles start at multiples of 4, hold
  at most the row cap, and their nonzeros fit the stage unless a tile is one
  group of 4 rows;
* each tile's cost is the number of distinct 32-byte sectors its gathers
  touch, counted here with numpy;
* the deal hands every tile to exactly one slot, keeps a round-robin deal's
  tile count per block and each block's tiles in table order, equals a
  restatement of its rule (heaviest first, to the least-loaded block with
  room, ties to the lower block), never leaves the heaviest block heavier
  than round-robin does on the bench's LP family, and is the identity for
  one block;
* the same input gives the same bytes twice.
"""
import heapq
import os
import shutil
import subprocess

import numpy as np
import pytest

from noaidi_b200.prima import generators as G

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(ROOT, "noaidi_b200", "csrc")
CAP32, CAP64, ROWS = 2048, 1536, 512


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if not cxx:
        pytest.skip("no host C++ compiler")
    exe = str(tmp_path_factory.mktemp("tiles") / "tile_deal_check")
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", CSRC, os.path.join(HERE, "tile_deal_check.cpp"),
                    os.path.join(CSRC, "prima_tiles.cpp"), "-o", exe], check=True)
    return exe


def run(exe, rp, ci, cols, cap, max_rows, word, nb):
    rows = len(rp) - 1
    blob = np.array([rows, cols, cap, max_rows, word, nb], dtype=np.int64).tobytes() + \
        np.asarray(rp, dtype=np.int32).tobytes() + np.asarray(ci, dtype=np.int32).tobytes()
    out = subprocess.run([exe], input=blob, capture_output=True, check=True).stdout
    nt = int(np.frombuffer(out[:8], dtype=np.int64)[0])
    o = 8
    table = np.frombuffer(out[o:o + 8 * (nt + 1)], dtype=np.int32).reshape(-1, 2)
    o += 8 * (nt + 1)
    cost = np.frombuffer(out[o:o + 4 * nt], dtype=np.float32)
    o += 4 * nt
    pairs = np.frombuffer(out[o:o + 16 * nt], dtype=np.int32).reshape(-1, 4)
    return table, cost, pairs, out


def sectors(table, rp, ci, word):
    shift = 2 if word == 8 else 3
    return np.array([len(np.unique(np.asarray(ci[rp[a]:rp[b]]) >> shift))
                     for a, b in zip(table[:-1, 0], table[1:, 0])], dtype=np.float32)


def deal_restated(cost, nb):
    """The deal's rule, restated: tiles heaviest first (stable), each to the
    least-loaded block with room (ties to the lower block); block b gets the
    round-robin count; slot b + k*nb is block b's k-th tile in table order."""
    nt = len(cost)
    if nb <= 1 or nt <= nb:
        return list(range(nt))
    order = sorted(range(nt), key=lambda j: -cost[j])
    room = [nt // nb + (1 if b < nt % nb else 0) for b in range(nb)]
    heap = [(0.0, b) for b in range(nb)]
    mine = [[] for _ in range(nb)]
    for j in order:
        load, b = heapq.heappop(heap)
        mine[b].append(j)
        room[b] -= 1
        if room[b] > 0:
            heapq.heappush(heap, (load + float(cost[j]), b))
    slot = [0] * nt
    for b in range(nb):
        for k, j in enumerate(sorted(mine[b])):
            slot[b + k * nb] = j
    return slot


def matrices():
    p = G.dc_lopf(seed=3, buses=120, lines=180, generators=60, snapshots=6)
    K = p.constraint_matrix
    yield "lopf-K", K.row_ptr, K.col_indices, K.cols
    Kt = K.transpose
    yield "lopf-Kt", Kt.row_ptr, Kt.col_indices, Kt.cols
    rng = np.random.default_rng(7)
    rows, cols = 5000, 3000
    lens = rng.integers(0, 9, rows)
    lens[rng.integers(0, rows, 6)] = rng.integers(700, 2600, 6)  # a few long rows
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = np.concatenate([np.sort(rng.choice(cols, int(n), replace=False)) for n in lens]).astype(np.int32)
    yield "random-long-rows", rp, ci, cols


@pytest.mark.parametrize("word,cap", [(4, CAP32), (8, CAP64)], ids=["fp32", "fp64"])
@pytest.mark.parametrize("max_rows", [ROWS, ROWS // 2])
def test_tile_table_and_costs(driver, word, cap, max_rows):
    for name, rp, ci, cols in matrices():
        table, cost, _, _ = run(driver, rp, ci, cols, cap, max_rows, word, 1)
        rows = len(rp) - 1
        assert table[0, 0] == 0 and table[-1, 0] == rows and table[-1, 1] == rp[-1], name
        starts, ends = table[:-1, 0], table[1:, 0]
        assert np.all(ends > starts) and np.all(starts % 4 == 0), name
        assert np.all(table[:, 1] == np.asarray(rp)[table[:, 0]]), name
        assert np.all(ends - starts <= max_rows), name
        span = ((np.asarray(rp)[ends].astype(np.int64) + 3) & ~3) - (np.asarray(rp)[starts] & ~3)
        assert np.all((span <= cap) | (ends - starts <= 4)), name
        np.testing.assert_array_equal(cost, sectors(table, rp, ci, word), err_msg=name)


@pytest.mark.parametrize("nb", [1, 7, 64, 444])
def test_deal_hands_out_every_tile_by_its_rule(driver, nb):
    for name, rp, ci, cols in matrices():
        table, cost, pairs, out = run(driver, rp, ci, cols, CAP32, ROWS, 4, nb)
        nt = len(cost)
        # each slot's pair is a tile's (start, end)
        index = {int(r): j for j, r in enumerate(table[:-1, 0])}
        slot_tile = [index[int(r)] for r in pairs[:, 0]]
        assert sorted(slot_tile) == list(range(nt)), name
        for s, j in enumerate(slot_tile):
            assert tuple(pairs[s]) == (*table[j], *table[j + 1]), name
        assert slot_tile == deal_restated(cost, nb), name
        # round-robin counts per block, tiles in table order within a block
        for b in range(min(nb, nt)):
            mine = slot_tile[b::nb]
            assert len(mine) == len(range(b, nt, nb)) and mine == sorted(mine), name
        # the same input, the same bytes
        assert run(driver, rp, ci, cols, CAP32, ROWS, 4, nb)[3] == out, name


def test_deal_balances_the_bench_family_at_least_as_well_as_round_robin(driver):
    p = G.dc_lopf(seed=0, buses=400, lines=600, generators=200, snapshots=24)
    for A in (p.constraint_matrix, p.constraint_matrix.transpose):
        for nb in (64, 148, 444):
            table, cost, pairs, _ = run(driver, A.row_ptr, A.col_indices, A.cols, CAP32, ROWS, 4, nb)
            nt = len(cost)
            index = {int(r): j for j, r in enumerate(table[:-1, 0])}
            slot_tile = np.array([index[int(r)] for r in pairs[:, 0]])
            dealt = np.bincount(np.arange(nt) % nb, weights=cost[slot_tile], minlength=nb)
            rr = np.bincount(np.arange(nt) % nb, weights=cost, minlength=nb)
            assert dealt.max() <= rr.max() + 1e-3, (nb, dealt.max(), rr.max())
