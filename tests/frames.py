"""Frame-reading helpers for tests: the form of a PRZM frame's Section 3."""
from __future__ import annotations


def section3_form(fr: bytes) -> str:
    """'stored' (uncompressed frame), 'empty', '09' (flat varints), '00'
    (flat 0x00 + LE32), or the distance-prefix header byte with the code
    stream's kind: '0B-M12', '0A-AD', ... (M12: Mode 12, AD: adaptive V-ANS)."""
    if len(fr) < 8 or fr[4] & 0x04:
        return "stored"
    if fr[4] & 0x08:
        l2 = fr[8] | fr[9] << 8 | fr[10] << 16
        l3 = fr[11] | fr[12] << 8 | fr[13] << 16
        w = 8 + 6 + 8 + l2
    else:
        l2 = fr[8] | fr[9] << 8
        l3 = fr[10] | fr[11] << 8
        w = 8 + 4 + 8 + l2
    if l3 == 0:
        return "empty"
    h = fr[w]
    if h in (0x00, 0x09):
        return "%02X" % h
    hl = {0x0B: 4, 0x0A: 7, 0x06: 13}[h]
    cs = fr[w + hl]
    return "%02X-%s" % (h, "M12" if cs == 0x0C else "AD" if cs == ord("V") else "?")


def section4_form(fr: bytes) -> str:
    """'stored', 'raw', 'AD' (adaptive V-ANS container) or 'SH<mode>' (an
    étale-sheaf container of that foliation)."""
    if len(fr) < 8 or fr[4] & 0x04:
        return "stored"
    if fr[4] & 0x08:
        l2 = fr[8] | fr[9] << 8 | fr[10] << 16
        l3 = fr[11] | fr[12] << 8 | fr[13] << 16
        w = 8 + 6 + 8 + l2 + l3
    else:
        l2 = fr[8] | fr[9] << 8
        l3 = fr[10] | fr[11] << 8
        w = 8 + 4 + 8 + l2 + l3
    if not fr[4] & 0x80:
        return "raw"
    f = fr[w + 3]
    return "SH%d" % (f >> 4) if f & 0x04 else "AD"
