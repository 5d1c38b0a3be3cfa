"""CPU check of the repeated-hash filter of the parallel-row and
parallel-column rules (gpu-preprocessor-ijoc_b200/csrc/rules_parallel.cu,
`mark_hash_bits` / `flag_repeated`), restated in numpy: every live item whose
hash another live item shares passes the filter, so the groups of two or more
that the (hash, index) sort finds among the passing items are exactly those
of the unfiltered sort, in the same order; and few unique hashes pass."""
import numpy as np
import pytest

M64 = (1 << 64) - 1


def mix(z):
    # SplitMix64 finaliser (the same mixing as the kernel's mix_hash).
    z = np.uint64(z)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def filter_flags(hashes, keep):
    n = len(hashes)
    lg = 20
    while lg < 29 and (1 << lg) < 32 * n:
        lg += 1
    mask = np.uint64((1 << lg) - 1)
    seen = np.zeros(1 << lg, dtype=bool)
    twice = np.zeros(1 << lg, dtype=bool)
    z = mix(hashes)
    b0, b1 = (z & mask).astype(np.int64), ((z >> np.uint64(32)) & mask).astype(np.int64)
    for i in np.random.default_rng(7).permutation(n):      # arrival order does not matter
        if not keep[i]:
            continue
        for b in (b0[i], b1[i]):
            if seen[b]:
                twice[b] = True
            seen[b] = True
    return keep & twice[b0] & twice[b1]


def groups(hashes, ids):
    order = np.lexsort((ids, hashes))      # stable sort by hash, ids ascending
    h, i = hashes[order], ids[order]
    out, start = [], 0
    for k in range(1, len(h) + 1):
        if k == len(h) or h[k] != h[start]:
            if k - start >= 2:
                out.append((int(h[start]), tuple(int(x) for x in i[start:k])))
            start = k
    return out


@pytest.mark.parametrize("seed", range(8))
def test_filter_keeps_every_group_whole_and_in_order(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(40_000, 120_000))
    hashes = rng.integers(0, 1 << 63, size=n, dtype=np.uint64)
    # Plant groups of equal hashes (parallel rows or columns).
    for _ in range(n // 50):
        size = int(rng.integers(2, 6))
        members = rng.choice(n, size=size, replace=False)
        hashes[members] = hashes[members[0]]
    keep = rng.random(n) < 0.9
    ids = np.arange(n)
    flags = filter_flags(hashes, keep)
    assert groups(hashes[keep], ids[keep]) == groups(hashes[flags], ids[flags])
    counts = {}
    for h in hashes[keep]:
        counts[int(h)] = counts.get(int(h), 0) + 1
    unique_passing = sum(1 for h, f in zip(hashes, flags) if f and counts[int(h)] == 1)
    assert unique_passing <= 0.01 * keep.sum()
