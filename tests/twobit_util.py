"""Writes UCSC .2bit files for the tests (seq/twobit.rs reads them): N runs become N blocks,
lower case becomes mask blocks, as faToTwoBit writes them."""
import struct

import numpy as np

_CODE = {ord("T"): 0, ord("C"): 1, ord("A"): 2, ord("G"): 3}


def _runs(flags: np.ndarray):
    d = np.diff(np.concatenate([[0], flags.astype(np.int8), [0]]))
    starts = np.nonzero(d == 1)[0]
    ends = np.nonzero(d == -1)[0]
    return list(zip(starts.tolist(), (ends - starts).tolist()))


def write_twobit(path, records, big_endian=False):
    """records: (name, ASCII sequence of ACGTN, either case)."""
    e = ">" if big_endian else "<"
    head = struct.pack(e + "IIII", 0x1A412743, 0, len(records), 0)
    index_size = sum(1 + len(n) + 4 for n, _ in records)
    blobs = []
    for name, seq in records:
        s = np.frombuffer(bytes(seq), dtype=np.uint8)
        upper = s & 0xDF
        nruns = _runs(upper == ord("N"))
        mruns = _runs(s != upper)
        codes = np.array([_CODE.get(int(c), 0) for c in upper], dtype=np.uint8)
        pad = (-len(codes)) % 4
        c4 = np.concatenate([codes, np.zeros(pad, np.uint8)]).reshape(-1, 4)
        packed = ((c4[:, 0] << 6) | (c4[:, 1] << 4) | (c4[:, 2] << 2) | c4[:, 3]).astype(np.uint8).tobytes()
        b = struct.pack(e + "II", len(s), len(nruns))
        b += b"".join(struct.pack(e + "I", st) for st, _ in nruns) + b"".join(struct.pack(e + "I", n) for _, n in nruns)
        b += struct.pack(e + "I", len(mruns))
        b += b"".join(struct.pack(e + "I", st) for st, _ in mruns) + b"".join(struct.pack(e + "I", n) for _, n in mruns)
        b += struct.pack(e + "I", 0) + packed
        blobs.append(b)
    off = len(head) + index_size
    index = b""
    for (name, _), b in zip(records, blobs):
        index += bytes([len(name)]) + name.encode() + struct.pack(e + "I", off)
        off += len(b)
    with open(path, "wb") as f:
        f.write(head + index + b"".join(blobs))


def read_twobit_ascii(data: bytes) -> list[tuple[str, bytes]]:
    """(name, upper-case ASCII sequence with its N blocks as N) per record of a UCSC .2bit image
    (either byte order); mask blocks are ignored.  For query fixtures kept as .2bit."""
    magic = struct.unpack("<I", data[:4])[0]
    e = "<" if magic == 0x1A412743 else ">"
    _, _, count, _ = struct.unpack(e + "IIII", data[:16])
    pos, index = 16, []
    for _ in range(count):
        ln = data[pos]
        name = data[pos + 1:pos + 1 + ln].decode()
        off = struct.unpack(e + "I", data[pos + 1 + ln:pos + 5 + ln])[0]
        index.append((name, off))
        pos += 5 + ln
    letters = np.frombuffer(b"TCAG", dtype=np.uint8)
    out = []
    for name, off in index:
        size, nb = struct.unpack(e + "II", data[off:off + 8])
        p = off + 8
        ns = np.frombuffer(data, dtype=e + "u4", count=nb, offset=p)
        nl = np.frombuffer(data, dtype=e + "u4", count=nb, offset=p + 4 * nb)
        p += 8 * nb
        mb = struct.unpack(e + "I", data[p:p + 4])[0]
        p += 4 + 8 * mb + 4
        packed = np.frombuffer(data, dtype=np.uint8, count=(size + 3) // 4, offset=p)
        codes = np.stack([(packed >> 6) & 3, (packed >> 4) & 3, (packed >> 2) & 3, packed & 3], axis=1).ravel()[:size]
        seq = letters[codes]
        for st, n in zip(ns.tolist(), nl.tolist()):
            seq[st:st + n] = ord("N")
        out.append((name, seq.tobytes()))
    return out
