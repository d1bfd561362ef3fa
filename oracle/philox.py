"""CPU restatement of the control variate's field-feature sampler (TEST
INFRASTRUCTURE ONLY: used by tests/ to check nrcps_cv_sample_z2_features,
never by the product path).

Philox4x32-10 is the counter-based generator of Salmon, Moraes, Dror and
Shaw, "Parallel random numbers: as easy as 1, 2, 3" (SC'11): ten rounds of
two 32x32->64-bit products (multipliers 0xD2511F53, 0xCD9E8D57) with the key
bumped by the Weyl constants (0x9E3779B9, 0xBB67AE85) between rounds.  It is
pinned by the known-answer vectors published with the authors' Random123
library (PHILOX_KATS below).

The sampler draws the block means of a uniform Z2 field directly: a cell of
n = (L/G)^3 sites has mean (2 c - n)/n with c = the number of set bits among
n independent fair bits, which is the exact distribution of the block mean
of n independent phi = +-1 sites.  The n bits of cell
g = ((first + b) T + t) G^3 + q are words 0..ceil(n/32)-1 of the cell, word
i being output i % 4 of the Philox call with counter
(lo32 g, hi32 g, i // 4, 0x5A32) and key (lo32 seed, hi32 seed); the last
word keeps its n mod 32 low bits.
"""
from __future__ import annotations

import numpy as np

M0, M1 = 0xD2511F53, 0xCD9E8D57
W0, W1 = 0x9E3779B9, 0xBB67AE85
TAG = 0x5A32

# (counter, key, output) of the Random123 known-answer file, philox4x32 with 10 rounds
PHILOX_KATS = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Vectorised over numpy arrays of uint32 (any broadcastable shapes)."""
    c = [np.asarray(v, dtype=np.uint64) for v in (c0, c1, c2, c3)]
    k0 = np.asarray(k0, dtype=np.uint64)
    k1 = np.asarray(k1, dtype=np.uint64)
    m32 = np.uint64(0xFFFFFFFF)
    for _ in range(10):
        p0 = np.uint64(M0) * c[0]
        p1 = np.uint64(M1) * c[2]
        c = [(p1 >> np.uint64(32)) ^ c[1] ^ k0, p1 & m32, (p0 >> np.uint64(32)) ^ c[3] ^ k1, p0 & m32]
        k0 = (k0 + np.uint64(W0)) & m32
        k1 = (k1 + np.uint64(W1)) & m32
    return [v.astype(np.uint32) for v in c]


def _popcount32(w: np.ndarray) -> np.ndarray:
    w = w.astype(np.uint64)
    w = w - ((w >> np.uint64(1)) & np.uint64(0x55555555))
    w = (w & np.uint64(0x33333333)) + ((w >> np.uint64(2)) & np.uint64(0x33333333))
    w = (w + (w >> np.uint64(4))) & np.uint64(0x0F0F0F0F)
    return ((w * np.uint64(0x01010101)) & np.uint64(0xFFFFFFFF)) >> np.uint64(24)


def z2_block_features(seed: int, first: int, L: int, T: int, G: int, B: int) -> np.ndarray:
    """Features [B, T, G^3] as FP32 values of the BF16 the device writes."""
    from .cvnet import to_bf16
    n = (L // G) ** 3
    GS = G ** 3
    g = (np.uint64(first) * np.uint64(T * GS) + np.arange(B * T * GS, dtype=np.uint64))
    lo = (g & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    hi = (g >> np.uint64(32)).astype(np.uint32)
    k0, k1 = np.uint32(seed & 0xFFFFFFFF), np.uint32((seed >> 32) & 0xFFFFFFFF)
    words = (n + 31) // 32
    cnt = np.zeros(g.shape, dtype=np.int64)
    for grp in range((words + 3) // 4):
        out = philox4x32_10(lo, hi, np.uint32(grp), np.uint32(TAG), k0, k1)
        for j in range(4):
            i = 4 * grp + j
            if i >= words:
                break
            w = out[j].astype(np.uint64)
            rem = n - 32 * i
            if rem < 32:
                w &= np.uint64((1 << rem) - 1)
            cnt += _popcount32(w).astype(np.int64)
    val = (2 * cnt - n).astype(np.float32) * (np.float32(1.0) / np.float32(n))
    return to_bf16(val).reshape(B, T, GS)
