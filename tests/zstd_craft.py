"""Hand-built zstd frames for the decoder's error paths (RFC 8878), shared by the host and GPU
zstd tests."""
from __future__ import annotations


def huf_tree_256_weights() -> bytes:
    """A Huffman tree description (RFC 8878 4.2.1) whose FSE-coded weights run to 256 entries.

    Header byte 36 (< 128: FSE-compressed weights, 36 bytes follow).  Distribution: accuracy
    log 5, symbols 0 and 1 with 16 states each, so every state reads exactly one bit
    (nb = 5 - highbit(16..31) = 1).  Coded as 4 bits (log - 5 = 0), 5 bits of 17 (count + 1,
    short form since 17 < 30) and 5 bits of 31 (long form: 31 - 14 = 17): 0x3F10, two bytes.
    The backward bit stream is 34 bytes whose last is 0x01 (end marker at bit 0): 264 bits.
    The two initial states take 10 (the first state 3: symbol 1, base 0; the second state 0:
    symbol 0, base 0), then one bit per weight; all zero bits keep both states at 0 (symbol 0),
    so the weights are a single 1 and zeros, whose sum 1 is completed by an implied last
    weight.  The read after weight 255 (a first-state read) runs past the start and the second
    state adds weight 256: one more explicit weight than a tree can have (libzstd refuses more
    than 255), and the implied weight would be the 257th."""
    stream = bytes(32) + b"\x18\x01"  # bits 259 and 260 set: the first state reads 3
    ncount = bytes([0x10, 0x3F])
    body = ncount + stream
    assert len(body) == 36
    return bytes([len(body)]) + body


def frame_with_huf_tree(tree: bytes, regenerated: int = 100) -> bytes:
    """One single-segment frame of one compressed block whose literals section is Huffman-coded
    with the given tree description (one stream; the stream bytes after it are zeros) and no
    sequences."""
    streams = bytes(4)
    comp = len(tree) + len(streams)
    assert regenerated < 1024 and comp < 1024
    # literals header, size format 0: type 2 (compressed), one stream, 10-bit sizes
    lh = 2 | (0 << 2) | (regenerated << 4) | (comp << 14)
    lit = lh.to_bytes(3, "little") + tree + streams
    block = lit + b"\x00"  # sequences: none
    bh = 1 | (2 << 1) | (len(block) << 3)  # last block, compressed
    magic = (0xFD2FB528).to_bytes(4, "little")
    return magic + bytes([0x20, regenerated]) + bh.to_bytes(3, "little") + block
