"""The child hit mask of the wide-BVH node test (rt_traverse.cuh,
intersect_children), restated in numpy: forming it four children per 32-bit
word from the nodes' meta bytes gives the same mask as testing each child's
internal-node bit and building its bits one by one.

A child's meta byte, as the host and device builders write it
(rt_bvh.cpp, rt_bvh_gpu.cu): an internal child (imask bit set) has
(1 << 5) | (24 + slot); a leaf child the unary mask of its 1-3 triangles
<< 5 | the bit of its first triangle (first + count <= 24); an empty slot 0.
The GPU parity tests check the kernels themselves; this pins the bit algebra
over every octant and random nodes and hit patterns.
"""
import numpy as np


def random_node(rng):
    imask = 0
    meta = [0] * 8
    off = 0
    for s in range(8):
        kind = rng.integers(0, 3)
        if kind == 1:
            imask |= 1 << s
            meta[s] = (1 << 5) | (24 + s)
        elif kind == 2:
            cnt = int(rng.integers(1, 4))
            if off + cnt <= 24:
                meta[s] = ({1: 1, 2: 3, 3: 7}[cnt] << 5) | off
                off += cnt
    return imask, meta


def per_child(imask, meta, oct_, hit):
    node_bits, tri_bits = 0, 0
    for s in range(8):
        if meta[s] == 0 or not hit[s]:
            continue
        if (imask >> s) & 1:
            node_bits |= 1 << (24 + (s ^ oct_))
        else:
            tri_bits |= (meta[s] >> 5) << (meta[s] & 31)
    return node_bits | imask, tri_bits


def word_wise(imask, meta, oct_, hit):
    hits = 0
    for half in range(2):
        m = sum(meta[4 * half + b] << (8 * b) for b in range(4))
        inner = m & ((m << 1) & 0xFFFFFFFF) & 0x10101010
        idx4 = (m ^ ((inner >> 4) * oct_)) & 0x1F1F1F1F
        bits4 = (m >> 5) & 0x07070707
        for b in range(4):
            if hit[4 * half + b]:
                hits |= ((bits4 >> (8 * b)) & 0xFF) << ((idx4 >> (8 * b)) & 0xFF)
    hits &= 0xFFFFFFFF
    return (hits & 0xFF000000) | imask, hits & 0x00FFFFFF


def test_word_wise_hit_mask_equals_per_child_rule():
    rng = np.random.default_rng(11)
    for _ in range(4000):
        imask, meta = random_node(rng)
        hit = rng.integers(0, 2, 8).astype(bool)
        for oct_ in range(8):
            assert word_wise(imask, meta, oct_, hit) == per_child(imask, meta, oct_, hit)


def test_leaf_indices_never_look_internal():
    # bits 3 and 4 of the index are both set only from 24 up, and a leaf's
    # first triangle bit is at most 23
    for off in range(24):
        assert not ((off >> 3) & 1 and (off >> 4) & 1)
    for s in range(8):
        assert ((24 + s) >> 3) & 1 and ((24 + s) >> 4) & 1
