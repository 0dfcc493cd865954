"""TEST INFRASTRUCTURE ONLY: numpy restatement of the synthetic graph generators.

An independent second implementation of the graph construction that the
library does in C++ (hc_gen_kronecker / hc_gen_uniform, host and device
builders), written from the construction's definition with whole-array numpy
operations instead of per-row loops:

  * random numbers: draw(seed, stream, i) = mix(mix(seed ^ stream * golden) + i),
    mix = the SplitMix64 finaliser (Steele, Lea and Flood 2014);
  * R-MAT endpoints (A = .57, B = .19, C = .19; the quadrant rule of
    src/gapbs/generator.h:82-115), one 24-bit uniform per bit level, two levels
    per 64-bit draw;
  * a vertex-id permutation: four rounds of odd multiply + add and xorshift,
    each invertible modulo 2^scale (in place of the shuffle of
    src/gapbs/generator.h:53-63);
  * uniform (Erdos-Renyi) endpoints (src/gapbs/generator.h:65-80);
  * weights: int32 uniform in [1, 255] or fp32 uniform in (0, 1]
    (src/gapbs/generator.h:133-147);
  * the build of src/gapbs/builder.h:141-186 and :366-406: both directions of
    every pair, self-loops dropped, duplicates merged keeping the lightest
    weight, vertices relabelled by (degree descending, old id descending), rows
    sorted by new neighbour id.

It pins the library's generators (tests/test_gen_oracle.py compares the CSR
arrays bit for bit), and it lets bench.py's reference arm build the benchmark
graph and write the .sg/.wsg files that the reference's own code reads, with
no part of this project's library loaded in that process.
"""
from __future__ import annotations

import numpy as np

_U64 = np.uint64
_MASK32 = _U64(0xFFFFFFFF)
_GOLDEN = _U64(0x9E3779B97F4A7C15)
K_RMAT, K_WEIGHT, K_PERM, K_UNIFORM = 1, 2, 3, 4
W_NONE, W_I32, W_F32 = 0, 1, 2


def _mix(z):
    """SplitMix64 finaliser on a uint64 array (wrapping arithmetic)."""
    z = np.asarray(z, dtype=_U64)
    z = (z ^ (z >> _U64(30))) * _U64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> _U64(27))) * _U64(0x94D049BB133111EB)
    return z ^ (z >> _U64(31))


def _draw(seed: int, stream: int, i):
    with np.errstate(over="ignore"):
        base = _mix(np.array([_U64(seed) ^ (_U64(stream) * _GOLDEN)], dtype=_U64))[0]
        return _mix(base + np.asarray(i, dtype=_U64))


def _permutation(bits: int, seed: int):
    mask = _U64(0xFFFFFFFF) if bits >= 32 else _U64((1 << bits) - 1)
    shift = _U64(bits // 2 + 1)
    k = _draw(seed, K_PERM, np.arange(4, dtype=_U64))
    mul = (k & _MASK32) | _U64(1)
    add = k >> _U64(32)

    def perm(x):
        x = np.asarray(x, dtype=_U64)
        for r in range(4):
            x = ((x * mul[r] + add[r]) & _MASK32) & mask
            x = x ^ (x >> shift)
        return x & mask
    return perm


def rmat_pairs(scale: int, seed: int, e):
    """Endpoints (src, dst) of R-MAT pairs with ids e (uint64 array)."""
    e = np.asarray(e, dtype=_U64)
    a, b, c = np.float32(0.57), np.float32(0.19), np.float32(0.19)
    ab = np.float32(a + b)
    abc = np.float32(ab + c)
    inv24 = np.float32(1.0 / 16777216.0)
    words = (scale + 1) // 2
    s = np.zeros(len(e), dtype=_U64)
    d = np.zeros(len(e), dtype=_U64)
    for k in range(words):
        with np.errstate(over="ignore"):
            h = _draw(seed, K_RMAT, e * _U64(words) + _U64(k))
        for half in range(2):
            if 2 * k + half >= scale:
                break
            bits24 = ((h >> _U64(8)) if half else (h >> _U64(40))) & _U64(0xFFFFFF)
            r = bits24.astype(np.float32) * inv24
            low = r < ab
            s = s << _U64(1)
            d = d << _U64(1)
            d += (low & (r > a)).astype(_U64)
            s += (~low).astype(_U64)
            d += (~low & (r > abc)).astype(_U64)
    perm = _permutation(scale, seed)
    return perm(s), perm(d)


def uniform_pairs(scale: int, seed: int, e):
    h = _draw(seed, K_UNIFORM, e)
    mask = _U64((1 << scale) - 1)
    return (h & _MASK32) & mask, (h >> _U64(32)) & mask


def weight_bits(wtype: int, seed: int, e):
    """Weight of pair e as its 32-bit pattern (int32 value or fp32 bits)."""
    h = _draw(seed, K_WEIGHT, e)
    if wtype == W_I32:
        return (_U64(1) + h % _U64(255)).astype(np.uint32)
    f = ((h >> _U64(40)) + _U64(1)).astype(np.float32) * np.float32(1.0 / 16777216.0)
    return f.view(np.uint32)


def build(kind: str, scale: int, factor: int, seed: int, wtype: int = W_NONE, chunk: int = 1 << 24):
    """(index int64[N+1], neighbors int32[M], weights int32/float32[M] or None)."""
    n = 1 << scale
    num_pairs = factor << scale
    srcs, dsts, ws = [], [], []
    for lo in range(0, num_pairs, chunk):
        e = np.arange(lo, min(lo + chunk, num_pairs), dtype=_U64)
        s, d = rmat_pairs(scale, seed, e) if kind == "kronecker" else uniform_pairs(scale, seed, e)
        keep = s != d
        s, d, e = s[keep], d[keep], e[keep]
        srcs += [s, d]
        dsts += [d, s]
        if wtype != W_NONE:
            w = weight_bits(wtype, seed, e).astype(_U64)
            ws += [w, w]
    src = np.concatenate(srcs) if srcs else np.zeros(0, _U64)
    dst = np.concatenate(dsts) if dsts else np.zeros(0, _U64)
    del srcs, dsts
    w = np.concatenate(ws) if ws else np.zeros(len(src), _U64)
    del ws
    # Merge duplicates keeping the lightest weight: sort by (src, dst, weight
    # bits) and keep the first of each (src, dst) run.  Non-negative fp32
    # weights order like their bit patterns.
    wbits = 8 if wtype == W_I32 else (32 if wtype == W_F32 else 0)
    if 2 * scale + wbits <= 64:
        key = (src << _U64(scale + wbits)) | (dst << _U64(wbits)) | w
        del src, dst, w
        key.sort()
        pair = key >> _U64(wbits)
        first = np.ones(len(key), dtype=bool)
        first[1:] = pair[1:] != pair[:-1]
        key = key[first]
        del pair, first
        src = key >> _U64(scale + wbits)
        dst = (key >> _U64(wbits)) & _U64((1 << scale) - 1)
        w = key & _U64((1 << wbits) - 1) if wbits else np.zeros(len(key), _U64)
        del key
    else:
        order = np.lexsort((w, (src << _U64(32)) | dst))
        src, dst, w = src[order], dst[order], w[order]
        pair = (src << _U64(32)) | dst
        first = np.ones(len(pair), dtype=bool)
        first[1:] = pair[1:] != pair[:-1]
        src, dst, w = src[first], dst[first], w[first]
        del pair, first, order
    deg = np.bincount(src.astype(np.int64), minlength=n)
    # New id = rank by (degree descending, old id descending).
    order_v = np.lexsort((-np.arange(n, dtype=np.int64), -deg))
    rank = np.empty(n, dtype=_U64)
    rank[order_v] = np.arange(n, dtype=_U64)
    nsrc, ndst = rank[src], rank[dst]
    del src, dst
    key = (nsrc << _U64(32)) | ndst
    order = np.argsort(key, kind="stable")
    nbr = ndst[order].astype(np.int32)
    index = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(nsrc.astype(np.int64), minlength=n), out=index[1:])
    weights = None
    if wtype != W_NONE:
        wb = w[order].astype(np.uint32)
        weights = wb.view(np.int32) if wtype == W_I32 else wb.view(np.float32)
    return index, nbr, weights


def write_graph(path: str, index, nbr, weights=None):
    """.sg / .wsg file (src/graph.cuh:207-224): [int32 N][int64 M][int64 index[N+1]], then M int32
    neighbours (.sg) or M (int32 neighbour, fp32 weight) pairs (.wsg; int32 weights as floats)."""
    n, m = len(index) - 1, len(nbr)
    with open(path, "wb") as f:
        f.write(np.int32(n).tobytes())
        f.write(np.int64(m).tobytes())
        f.write(np.ascontiguousarray(index, dtype=np.int64).tobytes())
        if weights is None:
            f.write(np.ascontiguousarray(nbr, dtype=np.int32).tobytes())
            return
        step = 1 << 22
        for lo in range(0, m, step):
            hi = min(lo + step, m)
            pairs = np.empty(2 * (hi - lo), dtype=np.uint32)
            pairs[0::2] = nbr[lo:hi].view(np.uint32)
            pairs[1::2] = np.asarray(weights[lo:hi], dtype=np.float32).view(np.uint32)
            f.write(pairs.tobytes())
