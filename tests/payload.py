"""Decoder of the Analyse output frame, restating the consumer's reader
(crates/svpflow-core/src/metadata.rs:246-273 decode_vectors, :460-481 decode_region)."""
from __future__ import annotations

import numpy as np


def header(payload: bytes) -> list:
    return list(np.frombuffer(bytes(payload[:0x40]), dtype="<i4"))


def decode(payload) -> dict:
    """-> {'header': [...16], 'previous': array or None, 'current': array or None};
    arrays are structured (dx, dy, score, luma)."""
    b = bytes(payload)
    h = header(b)
    assert h[0] == 16 and h[1] == 0xA0, "bad magic"
    flags, gw, gh = h[2], h[12], h[13]
    count = gw * gh
    out = {"header": h, "previous": None, "current": None}
    off = 0x40
    for name, bit in (("previous", 1), ("current", 2)):
        if not flags & bit:
            continue
        marker = int(np.frombuffer(b[off:off + 4], dtype="<i4")[0])
        assert marker == 2 * count + 1, "bad region marker"
        raw = np.frombuffer(b[off + 4:off + 4 + 8 * count], dtype="<u4").reshape(count, 2)
        rot = ((raw[:, 0] >> 16) | (raw[:, 0] << 16)) & 0xFFFFFFFF  # rotate_right(16)
        rec = np.zeros(count, dtype=[("dx", "<i2"), ("dy", "<i2"), ("score", "<u4"), ("luma", "u1")])
        rec["dx"] = (rot & 0xFFFF).astype(np.uint16).view(np.int16)
        rec["dy"] = (rot >> 16).astype(np.uint16).view(np.int16)
        rec["score"] = raw[:, 1] & 0xFFFFFF
        rec["luma"] = raw[:, 1] >> 24
        out[name] = rec
        off += 4 + 8 * count
    return out


def first_difference(a, b) -> str:
    """Human-readable first mismatch between two payloads (for assertion messages)."""
    a, b = bytes(a), bytes(b)
    if len(a) != len(b):
        return f"length {len(a)} != {len(b)}"
    if a == b:
        return "equal"
    da, db = decode(a), decode(b)
    if da["header"] != db["header"]:
        return f"header {da['header']} != {db['header']}"
    gw = da["header"][12]
    msgs = []
    for name in ("previous", "current"):
        x, y = da[name], db[name]
        if x is None:
            continue
        bad = np.nonzero(x != y)[0]
        if len(bad):
            i = int(bad[0])
            msgs.append(f"{name}: {len(bad)} of {len(x)} vectors differ; first at block ({i % gw},{i // gw}): "
                        f"got {tuple(x[i])} want {tuple(y[i])}")
    return "; ".join(msgs)
