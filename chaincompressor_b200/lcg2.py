"""Pure-Python reader of the LCG2 v2 container directory.

Walks the layout documented in chaincompressor_b200/csrc/chain_format.h and returns,
per component, its encoding, record count, byte size and rANS chunking (used for
size reports and for the algorithmic byte counts of the benchmark's roofline).  It
checks structure only; decoding is the library's job.
"""
import struct

ENC = {0: "empty", 1: "tagged", 2: "fixed", 3: "raw"}


class Reader:
    def __init__(self, b, pos=0):
        self.b, self.pos = b, pos

    def take(self, n):
        if self.pos + n > len(self.b):
            raise ValueError("truncated container")
        v = self.b[self.pos:self.pos + n]
        self.pos += n
        return v

    def u(self, fmt):
        return struct.unpack("<" + fmt, self.take(struct.calcsize(fmt)))[0]


def _section(r, count):
    prec, alphabet, tlen = r.u("B"), r.u("I"), r.u("I")
    r.take(tlen)
    S, lanes, chunks, payload = r.u("Q"), r.u("B"), r.u("I"), r.u("Q")
    lens = struct.unpack("<%dI" % chunks, r.take(4 * chunks))
    if sum(lens) != payload:
        raise ValueError("chunk lengths do not add up to the payload length")
    state_bytes = (lanes * chunks * (prec + 10) + 7) // 8   # final states, prec + 10 bits each
    r.take(state_bytes)
    r.take(payload)
    return {"prec": prec, "alphabet": alphabet, "table_bytes": tlen, "S": S, "lanes": lanes, "chunks": chunks,
            "payload": sum(lens), "symbols": count, "state_bytes": state_bytes}


def _component(r, body_len):
    start = r.pos
    enc, dims, records = r.u("B"), r.u("I"), r.u("Q")
    c = {"enc": ENC[enc], "dims": dims, "records": records, "bytes": body_len}
    if enc == 2:
        widths = []
        for _ in range(dims):
            r.u("Q")
            widths.append(r.u("B"))
        for w in widths:
            r.take((records * w + 7) // 8)
        c["widths"] = widths
    elif enc == 1:
        c["max_width"] = r.u("B")
        c["section"] = _section(r, records)
        bits = r.u("Q")
        r.take((bits + 7) // 8)
        c["packed_bits"] = bits
    elif enc == 3:
        c["section"] = _section(r, records * dims)
    if r.pos - start != body_len:
        raise ValueError("component length mismatch")
    return c


def inspect(data: bytes) -> dict:
    r = Reader(data)
    if r.take(4) != b"LCG2" or r.u("I") != 2:
        raise ValueError("not an LCG2 v2 container")
    D, N, p, eb, wmin, wmax = r.u("I"), r.u("Q"), r.u("q"), r.u("d"), r.u("q"), r.u("q")
    mins = [r.u("d") for _ in range(D)]
    dtype = r.u("B")
    assert r.u("I") == 5
    comps = {}
    for name in ("IDR0", "DIF0", "KEP0", "CH20", "REL0"):
        assert r.take(4).decode() == name
        comps[name] = _component(r, r.u("Q"))
    assert r.take(4) == b"EXC0"
    exc_len = r.u("Q")
    exc_start = r.pos
    count = r.u("Q")
    exc = {"count": count, "bytes": exc_len}
    if count:
        nd = r.u("Q")
        r.take(8 * nd)
        exc["distinct"] = nd
        exc["gaps"] = _component(r, r.u("Q"))
        exc["ids"] = _component(r, r.u("Q"))
    assert r.pos == exc_start + exc_len == len(data)
    return {"D": D, "N": N, "p": p, "eb": eb, "wrap": (wmin, wmax), "mins": mins, "input_dtype": dtype,
            "components": comps, "corrections": exc, "bytes": len(data)}
