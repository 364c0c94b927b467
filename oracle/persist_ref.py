"""Restatement of the versioned model container written by tm_save.

TEST INFRASTRUCTURE ONLY (the checker for tm_save / tm_save_buf and the
container branch of tm_load).  The container wraps the reference's own
persisted record (capi.c:1509-1531: type, thirteen u32 fields, specificity,
tail mask, actions, individualized flag, feature sizes) unchanged, and adds
what that record lacks: a format version, `negative`, the default seed, the
reusable flag and, optionally, the count planes (capi.c:1696 drops them).

Layout, little-endian:
    "STMV" | u32 version=1 | u32 flags (1 state, 2 reusable) | u32 0 |
    f64 negative | u64 seed | u64 record_len | record |
    [u64 state_len | state] | u64 FNV-1a 64 of all preceding bytes
"""
import struct

MAGIC = b"STMV"
VERSION = 1


def fnv1a64(data):
    """FNV-1a, 64-bit (Fowler, Noll, Vo): offset basis 0xcbf29ce484222325,
    prime 0x100000001b3."""
    h = 0xCBF29CE484222325
    for b in data:
        h ^= b
        h = (h * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


def container(record, state=None, negative=0.0, seed=0, reusable=False, version=VERSION):
    flags = (1 if state is not None else 0) | (2 if reusable else 0)
    out = bytearray(MAGIC)
    out += struct.pack("<III", version, flags, 0)
    out += struct.pack("<dQQ", float(negative), int(seed), len(record))
    out += bytes(record)
    if state is not None:
        out += struct.pack("<Q", len(state)) + bytes(state)
    out += struct.pack("<Q", fnv1a64(out))
    return bytes(out)


def parse(blob):
    """(version, flags, negative, seed, record, state or None); raises
    ValueError on a bad magic or checksum."""
    if blob[:4] != MAGIC:
        raise ValueError("not a container")
    if fnv1a64(blob[:-8]) != struct.unpack("<Q", blob[-8:])[0]:
        raise ValueError("checksum mismatch")
    version, flags, _ = struct.unpack("<III", blob[4:16])
    negative, seed, rl = struct.unpack("<dQQ", blob[16:40])
    record = blob[40:40 + rl]
    state = None
    if flags & 1:
        (sl,) = struct.unpack("<Q", blob[40 + rl:48 + rl])
        state = blob[48 + rl:48 + rl + sl]
    return version, flags, negative, seed, record, state
