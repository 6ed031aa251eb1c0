"""A second, pure-Python restatement of the match finders and the tokenizer
(gpu/kernel/przm_lz77.cu:156-360, gpu/kernel/przm_tokenizer.cuh:115-466),
written independently of oracle/przm_oracle.c so the two cross-check each
other.  Slow: small inputs only.  Test infrastructure."""
from __future__ import annotations

import numpy as np

MASK32 = 0xFFFFFFFF
MASK64 = (1 << 64) - 1


def _u32(b: bytes, i: int) -> int:
    return int.from_bytes(b[i:i + 4], "little")


def _pack(length: int, off: int) -> int:
    if length < 4 or off == 0:
        return 0
    return (min(length, 4095) << 20) | (off & 0xFFFFF)


def _lcp(b: bytes, p: int, c: int, limit: int) -> int:
    k = 0
    while k < limit and b[p + k] == b[c + k]:
        k += 1
    return k


def tile_find(a: np.ndarray) -> np.ndarray:
    b = bytes(a)
    n = len(b)
    out = np.zeros(n, np.uint32)
    for ts in range(0, n, 32768):
        t = b[ts:ts + 32768]
        tl = len(t)
        head = [0] * 2048
        for st in range(0, tl, 256):
            ps = range(st, min(st + 256, tl))
            w = {p: _u32(t, p) for p in ps if p + 4 <= tl}
            h = {p: ((w[p] * 0x1E35A7BD) & MASK32) >> 21 & 2047 for p in w}
            for p in ps:
                if p not in w:
                    out[ts + p] = 0
                    continue
                lim = min(tl - p, 4095)
                lane = (p - st) & 31
                best_len = best_off = 0
                for dlt in range(1, 5):
                    if lane >= dlt and w[p - dlt] == w[p]:
                        L = _lcp(t, p, p - dlt, lim)
                        if L > best_len:
                            best_len, best_off = L, dlt
                v = head[h[p]]
                for k, c16 in enumerate((v >> 16, v & 0xFFFF)):
                    if c16 == 0 or (k == 1 and best_len >= 258):
                        continue
                    c = c16 - 1
                    if c < p and _u32(t, c) == w[p]:
                        L = _lcp(t, p, c, lim)
                        if L > best_len:
                            best_len, best_off = L, p - c
                out[ts + p] = _pack(best_len, best_off) if best_len >= 4 else 0
            for p in ps:  # ascending insertion
                if p in w:
                    head[h[p]] = ((p + 1) << 16) | (head[h[p]] >> 16)
    return out


def radix_find(a: np.ndarray) -> np.ndarray:
    b = bytes(a)
    n = len(b)
    out = np.zeros(n, np.uint32)
    last: dict[int, int] = {}
    for p in range(0, n - 7, 8):
        k = int.from_bytes(b[p:p + 8], "little")
        h = ((k * 0x9E3779B97F4A7C15) & MASK64) >> 43 & ((1 << 19) - 1)
        q = last.get(h)
        last[h] = p
        if q is None:
            continue
        d = p - q
        if d > 1048575 or b[q:q + 8] != b[p:p + 8]:
            continue
        L = 8 + _lcp(b, p + 8, q + 8, min(n - p - 8, 4095 - 8))
        out[p] = _pack(L, d)
    return out


def _varint(v: int) -> bytes:
    o = bytearray()
    while v >= 0x80:
        o.append((v & 0x7F) | 0x80)
        v >>= 7
    o.append(v)
    return bytes(o)


def _litop(count: int) -> bytes:
    if count == 0:
        return b""
    if count <= 8:
        return bytes([0xF2 + count])
    return bytes([0xF0]) + _varint(count)


def tokenize(a: np.ndarray, desc: np.ndarray) -> tuple[bytes, bytes, bytes]:
    b = bytes(a)
    n = len(b)
    cmd, off, lit = bytearray(), bytearray(), bytearray()
    for start in range(0, n, 32768):
        end = min(start + 32768, n)
        rep = [1, 4, 8] if start == 0 else [-1, -1, -1]
        pos = ls = start
        while pos < end:
            q = pos
            while q < end and desc[q] == 0:
                q += 1
            if q >= end:
                break
            m, d = int(desc[q]) >> 20, int(desc[q]) & 0xFFFFF
            if q + 1 < end and desc[q + 1] and (int(desc[q + 1]) >> 20) > m + 1:
                pos = q + 1
                continue
            if q + 12 <= end and b[q:q + 4] == bytes([b[q]]) * 4:
                r = 4
                while r < min(end - q, 65535) and b[q + r] == b[q]:
                    r += 1
                if r >= 12 and r >= m:
                    if q > ls:
                        cmd += _litop(q - ls)
                        lit += b[ls:q]
                    cmd += bytes([0xF1]) + _varint(r)
                    lit.append(b[q])
                    pos = ls = q + r
                    continue
            if not (0 < d <= q and m >= 4 and b[q:q + 4] == b[q - d:q - d + 4]):
                pos = q + 1
                continue
            m = min(m, end - q)
            while q + m < end and b[q + m] == b[q - d + m] and m < 65530:
                m += 1
            k = rep.index(d) if d in rep and d > 0 else -1
            ll = q - ls
            keep = (7 if m <= 7 else 15) if k >= 0 else 3
            if ll > keep:
                cmd += _litop(ll - keep)
                lit += b[ls:q - keep]
                ls, ll = q - keep, keep
            base = min(m - 4, 15)
            if k >= 0 and m <= 7:
                cmd.append((ll << 4) | ((m - 4) << 2) | k)
            elif k >= 0:
                cmd += bytes([0xC0 | k, (ll << 4) | base]) + (_varint(m - 19) if base == 15 else b"")
            else:
                cmd += bytes([0x80 | (ll << 4) | base]) + (_varint(m - 19) if base == 15 else b"")
            lit += b[ls:q]
            if k < 0:
                off += _varint(d)
                rep = [d, rep[0], rep[1]]
            elif k == 1:
                rep = [d, rep[0], rep[2]]
            elif k == 2:
                rep = [d, rep[0], rep[1]]
            pos = ls = q + m
        if ls < end:
            cmd += _litop(end - ls)
            lit += b[ls:end]
    return bytes(cmd), bytes(off), bytes(lit)
