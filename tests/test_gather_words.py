"""The float32 identities behind the stage kernels' gather words (csrc/swe_tiled.cuh).

The kernels store an edge's words as each of its cells adds them: the left cell adds
(w0, w1, w2), the right cell adds (-w0, -w3, -w4), and an edge that is not computed
(dry on both sides) holds -0.0 in every word. The reference's gather
(inundation/vulkan/shaders/resident.py:312-344) skips such edges and subtracts on the
right side instead. The two agree bit for bit under IEEE round-to-nearest without
flush to zero (the build's -ftz=false), because x + (-0.0) == x for every x, +0.0
included, and x + (-w) is x - w. These tests check both identities on float32 values,
signed zeros, subnormals and infinities included, and replay both gathers over random
tiles.
"""
import numpy as np

F32 = np.float32


def _bits(x):
    return np.asarray(x, dtype=np.float32).view(np.uint32)


def _specials():
    return np.array([0.0, -0.0, 1e-45, -1e-45, 1.1754942e-38, -1.1754942e-38, 1.0, -1.0, 3.4028235e38,
                     -3.4028235e38, np.inf, -np.inf], dtype=np.float32)


def test_adding_negative_zero_leaves_every_float_unchanged():
    rng = np.random.default_rng(5)
    x = np.concatenate([_specials(), rng.standard_normal(4096).astype(np.float32),
                        rng.integers(0, 2**32, 4096, dtype=np.uint64).astype(np.uint32).view(np.float32)])
    x = x[~np.isnan(x)]
    got = x + np.float32(-0.0)
    assert np.array_equal(_bits(got), _bits(x))
    # +0.0 would not do: -0.0 + +0.0 is +0.0
    assert _bits(np.float32(-0.0) + np.float32(0.0)) != _bits(np.float32(-0.0))


def test_adding_the_negation_is_subtracting():
    rng = np.random.default_rng(6)
    a = np.concatenate([_specials(), rng.standard_normal(4096).astype(np.float32) * 1e3])
    b = np.concatenate([_specials()[::-1], rng.standard_normal(4096).astype(np.float32)])
    with np.errstate(invalid="ignore", over="ignore"):
        sub = a - b
        add = a + (-b)
    ok = ~(np.isnan(sub) & np.isnan(add))
    assert np.array_equal(_bits(sub[ok]), _bits(add[ok]))
    assert np.array_equal(np.isnan(sub), np.isnan(add))


def _tile(rng, n_cells, n_edges):
    words = (rng.standard_normal((n_edges, 6)) * rng.choice([1e-6, 1.0, 1e3], (n_edges, 1))).astype(np.float32)
    words[rng.random(n_edges) < 0.1, 0] = np.float32(-0.0)  # signed zeros among the computed words
    live = rng.random(n_edges) < 0.6
    slots = [[] for _ in range(n_cells)]
    for j in range(n_edges):
        left, right = rng.choice(n_cells, 2, replace=False)
        slots[left].append(2 * j)
        slots[right].append(2 * j + 1)
    for s in slots:
        rng.shuffle(s)
    return words, live, slots


def _reference_gather(words, live, slots):
    out = []
    for s in slots:
        sdh = sdhu = sdhv = lam = F32(0.0)
        for v in s:
            j = v >> 1
            if not live[j]:
                continue
            w0, w1, w2, w3, w4, w5 = words[j]
            if v & 1:
                sdh, sdhu, sdhv = sdh - w0, sdhu - w3, sdhv - w4
            else:
                sdh, sdhu, sdhv = sdh + w0, sdhu + w1, sdhv + w2
            lam = lam + w5
        out.append((sdh, sdhu, sdhv, lam))
    return np.array(out, dtype=np.float32)


def _side_word_gather(words, live, slots):
    z = F32(-0.0)
    n_edges = len(words)
    slot = np.full((2 * n_edges, 4), z, dtype=np.float32)  # the persistent kernel's float4 slot words
    for j in range(n_edges):
        if live[j]:
            w0, w1, w2, w3, w4, w5 = words[j]
            slot[2 * j] = (w0, w1, w2, w5)
            slot[2 * j + 1] = (-w0, -w3, -w4, w5)
    out = []
    for s in slots:
        acc = [F32(0.0)] * 4
        for v in s:
            acc = [acc[k] + slot[v, k] for k in range(4)]
        out.append(acc)
    return np.array(out, dtype=np.float32)


def test_side_word_gather_has_the_bits_of_the_reference_gather():
    rng = np.random.default_rng(7)
    for _ in range(20):
        words, live, slots = _tile(rng, 64, 200)
        ref = _reference_gather(words, live, slots)
        got = _side_word_gather(words, live, slots)
        assert np.array_equal(_bits(got), _bits(ref))


def test_a_cell_with_only_dry_edges_keeps_positive_zero_sums():
    rng = np.random.default_rng(8)
    words, live, slots = _tile(rng, 16, 40)
    live[:] = False
    got = _side_word_gather(words, live, slots)
    assert np.all(_bits(got) == 0)  # +0.0, as the reference's untouched accumulators
