"""CPU checks of the index arithmetic of the single-pass compaction
(gpu-preprocessor-ijoc_b200/csrc/compact.cu), restated in numpy:

- the per-tile first-row map (`compact_tile_rows`) gives every tile exactly
  one value, the first row whose pointer is at or past the tile's start;
- the row of every stored entry follows from the row starts marked inside
  its tile (`tile_kept_mask`), empty rows included;
- every kept row's new pointer is written by exactly one tile, and the
  result equals a plain row-by-row compaction;
- the decoupled look-back (`tile_lookback`: windows of 32 predecessors, sums
  back to the nearest inclusive count) returns each tile's exclusive prefix
  whatever order the tiles publish in.

The GPU suite checks the kernels themselves against the oracle and the
reference; these tests pin the index logic on inputs the GPU tests do not
reach (tiny tiles, runs of empty rows, rows ending exactly on a tile edge)."""
import numpy as np
import pytest

PER = 8


def first_rows(ptr, tiles, tile):
    rows = len(ptr) - 1
    out = np.full(tiles, -1, dtype=np.int64)
    for r in range(rows + 1):
        lo = 0 if r == 0 else ptr[r - 1] // tile + 1
        hi = tiles - 1 if r == rows else min(ptr[r] // tile, tiles - 1)
        for t in range(lo, hi + 1):
            assert out[t] == -1, "a tile is assigned twice"
            out[t] = r
    assert (out >= 0).all(), "a tile is not assigned"
    return out


def compact(ptr, idx, outer, inner, tile):
    rows, nnz = len(ptr) - 1, int(ptr[-1])
    tiles = (nnz + tile - 1) // tile
    first = first_rows(ptr, tiles, tile)
    kept_tiles = []
    for t in range(tiles):
        base, ln = t * tile, min(tile, nnz - t * tile)
        r0, r1 = first[t], (first[t + 1] if t + 1 < tiles else rows)
        assert all(ptr[r] >= base for r in range(r0, r1))
        marks = np.zeros(tile, dtype=np.int64)
        for r in range(r0, r1):
            if ptr[r] - base < ln:
                marks[ptr[r] - base] += 1
        starts = np.cumsum(marks)
        kept = np.zeros(ln, dtype=bool)
        for q in range(ln):
            row = r0 - 1 + starts[q]
            assert 0 <= row < rows and ptr[row] <= base + q < ptr[row + 1]
            kept[q] = outer[row] >= 0 and inner[idx[base + q]] >= 0
        kept_tiles.append((kept, r0, r1, base, ln))
    offsets = np.concatenate([[0], np.cumsum([k.sum() for k, *_ in kept_tiles])])
    new_rows = int((outer >= 0).sum())
    out_ptr = np.full(new_rows + 1, -1, dtype=np.int64)
    out_idx = np.full(int(offsets[-1]), -1, dtype=np.int64)
    for t, (kept, r0, r1, base, ln) in enumerate(kept_tiles):
        before = np.concatenate([[0], np.cumsum(kept)])
        for q in np.nonzero(kept)[0]:
            out_idx[offsets[t] + before[q]] = inner[idx[base + q]]
        for r in range(r0, r1):
            if outer[r] < 0:
                continue
            pos = ptr[r] - base
            assert out_ptr[outer[r]] == -1, "a row pointer is written twice"
            out_ptr[outer[r]] = offsets[t] + (before[pos] if pos < ln else before[ln])
        if t == tiles - 1:
            out_ptr[new_rows] = offsets[t] + before[ln]
    return out_ptr, out_idx


def plain_compact(ptr, idx, outer, inner):
    out_ptr, out_idx = [0], []
    for r in range(len(ptr) - 1):
        if outer[r] < 0:
            continue
        out_idx += [inner[j] for j in idx[ptr[r]:ptr[r + 1]] if inner[j] >= 0]
        out_ptr.append(len(out_idx))
    return np.array(out_ptr), np.array(out_idx, dtype=np.int64)


def maps(keep):
    return np.where(keep, np.cumsum(keep) - 1, -1)


@pytest.mark.parametrize("seed", range(60))
def test_tiled_compaction_equals_row_compaction(seed):
    rng = np.random.default_rng(seed)
    tile = PER * int(rng.choice([1, 2, 4]))
    rows, cols = int(rng.integers(1, 50)), int(rng.integers(1, 30))
    lens = rng.integers(0, [3, 12, 40, 6][seed % 4] + 1, size=rows)
    if seed % 4 == 3:
        lens[rng.random(rows) < 0.7] = 0          # runs of empty rows
    if lens.sum() == 0:
        lens[-1] = 1
    ptr = np.concatenate([[0], np.cumsum(lens)])
    idx = rng.integers(0, cols, size=int(ptr[-1]))
    keep_r, keep_c = rng.random(rows) < rng.uniform(0.3, 1.0), rng.random(cols) < rng.uniform(0.3, 1.0)
    keep_r[0] = keep_c[0] = True
    got = compact(ptr, idx, maps(keep_r), maps(keep_c), tile)
    want = plain_compact(ptr, idx, maps(keep_r), maps(keep_c))
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


@pytest.mark.parametrize("lens", [[16, 0, 0], [8, 8, 0, 0], [0, 0, 16, 16, 0], [1] * 40, [0, 48], [5, 0, 0, 0, 11]])
def test_rows_on_tile_edges(lens):
    lens = np.array(lens)
    ptr = np.concatenate([[0], np.cumsum(lens)])
    idx = np.zeros(int(ptr[-1]), dtype=np.int64)
    keep_r = np.ones(len(lens), dtype=bool)
    got = compact(ptr, idx, maps(keep_r), np.array([0]), 16)
    want = plain_compact(ptr, idx, maps(keep_r), np.array([0]))
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


AGG, INCL = 1, 2


def lookback(status, t, window=32):
    """tile_lookback: read predecessors t-1, t-2, ... `window` at a time; sum
    their values back to (and including) the nearest inclusive count."""
    before, end = 0, t - 1
    while True:
        lanes = []
        for lane in range(window):
            j = end - lane
            lanes.append((INCL, 0) if j < 0 else status[j])
        assert all(flag != 0 for flag, _ in lanes), "a lane reads an unpublished tile"
        first = next((k for k, (flag, _) in enumerate(lanes) if flag == INCL), window)
        before += sum(v for k, (_, v) in enumerate(lanes) if k <= first)
        if first < window:
            return before
        end -= window


@pytest.mark.parametrize("seed", range(20))
def test_lookback_gives_exclusive_prefix_in_any_publication_order(seed):
    rng = np.random.default_rng(seed)
    tiles = int(rng.integers(1, 300))
    counts = rng.integers(0, 2048, size=tiles)
    truth = np.concatenate([[0], np.cumsum(counts)])
    status = [(0, 0)] * tiles
    # Tiles take tickets in order; each publishes its aggregate at once, and
    # its inclusive count after its look-back, at a random later moment.
    pending = []
    for t in range(tiles):
        status[t] = (INCL, int(counts[0])) if t == 0 else (AGG, int(counts[t]))
        if t > 0:
            pending.append(t)
        rng.shuffle(pending)
        while pending and rng.random() < 0.5:
            u = pending.pop()
            # A tile's look-back may only wait on predecessors (all published).
            b = lookback(status, u)
            assert b == truth[u]
            status[u] = (INCL, b + int(counts[u]))
    for u in pending:
        b = lookback(status, u)
        assert b == truth[u]
        status[u] = (INCL, b + int(counts[u]))
