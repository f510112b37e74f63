"""CPU restatement of the block-parameter coder and its predictor (test infrastructure only).

The extended container codes the repos / SFC-delta stream in blocks of 1024 values, each with
a PFor slot width w in 0..32 and a Golomb-Rice parameter k in 0..31 (the reference has no such
format: it codes this stream with one Golomb-Rice k for PFor patches and a Huffman code,
source/composer/block_compressor.hpp:122-136, 174-190).  This module restates, in numpy:

  * cost / exhaustive search / features / encoder / decoder of the block coder
    (xnyzip_b200/csrc/k_blocks.cu);
  * the 34-64-64-(32+33) predictor's forward pass, softmax cross-entropy loss and gradients,
    rounding to BF16 exactly where the tensor-core kernels do (xnyzip_b200/csrc/k_mlp.cu):
    weights, inputs, hidden activations and back-propagated gradients; sums in float64.

Only tests, the smoke entry point and the bench's CPU baseline may use it.
"""
from __future__ import annotations

import numpy as np

BLK = 1024
NF = 34
NI, NH, NO, NOP = 48, 64, 72, 80
NK, NW = 32, 33
OFF = {}
_o = 0
for _name, _size in (("W1", NH * NI), ("b1", NH), ("W2", NH * NH), ("b2", NH), ("W3", NO * NH), ("b3", NO)):
    OFF[_name] = (_o, _o + _size)
    _o += _size
NPARAM = _o


# ------------------------------------------------------------------- block coder ---------
def _bitlen(x: np.ndarray) -> np.ndarray:
    x = np.asarray(x, dtype=np.uint64)
    out = np.zeros(x.shape, dtype=np.int64)
    y = x.copy()
    for s in (32, 16, 8, 4, 2, 1):
        m = y >= (np.uint64(1) << np.uint64(s))
        out[m] += s
        y[m] >>= np.uint64(s)
    out[y > 0] += 1
    return out


def esc_len(e: np.ndarray, k: int) -> np.ndarray:
    q = np.asarray(e, dtype=np.uint64) >> np.uint64(k)
    return np.where(q < 32, q.astype(np.int64) + 1 + k, 97 + k)


def block_cost(v: np.ndarray, w: int, k: int) -> int:
    w, k = int(w), int(k)
    thr = np.uint64((1 << w) - 1)
    v = np.asarray(v, dtype=np.uint64)
    esc = v >= thr
    return int(v.size * w + esc_len(v[esc] - thr, k).sum())


def cost_table(v: np.ndarray) -> np.ndarray:
    """[33, 32] sizes in bits of one block for every (w, k)."""
    t = np.zeros((NW, NK), dtype=np.int64)
    for w in range(NW):
        for k in range(NK):
            t[w, k] = block_cost(v, w, k)
    return t


def search(vals: np.ndarray):
    """Exhaustive (w, k, cost) per block; ties: smallest w, then smallest k."""
    vals = np.asarray(vals, dtype=np.uint64)
    nb = (vals.size + BLK - 1) // BLK
    W = np.zeros(nb, np.uint8)
    K = np.zeros(nb, np.uint8)
    Cst = np.zeros(nb, np.int64)
    for b in range(nb):
        t = cost_table(vals[b * BLK:(b + 1) * BLK])
        i = int(np.argmin(t))  # row-major: smallest w first, then k
        W[b], K[b], Cst[b] = i // NK, i % NK, t.flat[i]
    return W, K, Cst


def features(vals: np.ndarray) -> np.ndarray:
    vals = np.asarray(vals, dtype=np.uint64)
    nb = (vals.size + BLK - 1) // BLK
    f = np.zeros((nb, NF), np.float32)
    for b in range(nb):
        x = vals[b * BLK:(b + 1) * BLK]
        bl = np.minimum(_bitlen(x), 31)
        f[b, :32] = np.bincount(bl, minlength=32)[:32] / x.size
        l = np.log2(x.astype(np.float32) + np.float32(1.0)).astype(np.float32)
        f[b, 32] = l.mean(dtype=np.float64) / 64.0
        f[b, 33] = l.max() / 64.0
    return f


class _Bits:
    def __init__(self):
        self.words = {}

    def put(self, pos: int, val: int, n: int):
        val &= (1 << n) - 1 if n < 64 else (1 << 64) - 1
        for i in range(n):
            if (val >> i) & 1:
                p = pos + i
                self.words[p >> 5] = self.words.get(p >> 5, 0) | (1 << (p & 31))

    def to_bytes(self, nbits: int) -> bytes:
        nw = (nbits + 31) // 32
        arr = np.zeros(nw, np.uint32)
        for k, v in self.words.items():
            if k < nw:
                arr[k] = v
        return arr.tobytes()[: (nbits + 7) // 8]


def encode(vals: np.ndarray, W: np.ndarray, K: np.ndarray):
    """(offsets, payload bytes, payload bits) of the block-coded stream.  Per block: w-bit
    slots, then the unary parts of the escapes (min(q, 32) ones and a zero each), their k-bit
    remainders, and the 64-bit values of the capped escapes (q >= 32)."""
    vals = [int(x) for x in np.asarray(vals, dtype=np.uint64)]
    nb = len(W)
    bits = _Bits()
    offs = np.zeros(nb, np.uint64)
    pos = 0
    for b in range(nb):
        offs[b] = pos
        x = vals[b * BLK:(b + 1) * BLK]
        w, k = int(W[b]), int(K[b])
        thr = (1 << w) - 1
        for i, v in enumerate(x):
            bits.put(pos + i * w, thr if v >= thr else v, w)
        pos += len(x) * w
        esc = [v - thr for v in x if v >= thr]
        for e in esc:  # U
            q = min(e >> k, 32)
            bits.put(pos, (1 << q) - 1, q + 1)
            pos += q + 1
        for e in esc:  # R
            bits.put(pos, e, k)
            pos += k
        for e in esc:  # X
            if e >> k >= 32:
                bits.put(pos, e, 64)
                pos += 64
    return offs, bits.to_bytes(pos), pos


def decode(payload: bytes, nbits: int, n: int, W, K, offs) -> np.ndarray:
    words = np.frombuffer(payload + b"\0" * 16, dtype=np.uint8)
    bitsarr = np.unpackbits(words, bitorder="little")

    def get(pos, m):
        v = 0
        for i in range(m):
            v |= int(bitsarr[pos + i]) << i
        return v

    out = np.zeros(n, np.uint64)
    for b in range(len(W)):
        cnt = min(BLK, n - b * BLK)
        w, k = int(W[b]), int(K[b])
        thr = (1 << w) - 1
        base = int(offs[b])
        slots = [get(base + i * w, w) if w else 0 for i in range(cnt)]
        pos = base + cnt * w
        qs = []
        for s in slots:
            if s != thr:
                continue
            q = 0
            while bitsarr[pos + q]:
                q += 1
            qs.append(q)
            pos += q + 1
        rems = []
        for _ in qs:
            rems.append(get(pos, k))
            pos += k
        j = 0
        for i, s in enumerate(slots):
            if s == thr:
                if qs[j] >= 32:
                    e = get(pos, 64)
                    pos += 64
                else:
                    e = (qs[j] << k) | rems[j]
                out[b * BLK + i] = thr + e
                j += 1
            else:
                out[b * BLK + i] = s
    return out


# ------------------------------------------------------------------- predictor -----------
def bf16(x) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    a = np.asarray(x, dtype=np.float32).copy()
    u = a.view(np.uint32)
    r = ((u >> 16) & 1) + np.uint32(0x7FFF)
    u[:] = (u + r) & np.uint32(0xFFFF0000)
    return a


def unpack(prm: np.ndarray):
    p = np.asarray(prm)
    g = lambda n: p[OFF[n][0]:OFF[n][1]]
    return (g("W1").reshape(NH, NI), g("b1"), g("W2").reshape(NH, NH), g("b2"), g("W3").reshape(NO, NH), g("b3"))


def init_params(seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, np.float32)
    for name, fan_in in (("W1", NF), ("W2", NH), ("W3", NH)):
        a, b = OFF[name]
        m = rng.normal(0.0, np.sqrt(2.0 / fan_in), b - a).astype(np.float32)
        if name == "W1":
            m = m.reshape(NH, NI)
            m[:, NF:] = 0.0
            m = m.ravel()
        if name == "W3":
            m = m.reshape(NO, NH)
            m[NK + NW:, :] = 0.0
            m = m.ravel()
        p[a:b] = m
    return p


def _rounder(exact: bool):
    if exact:
        return lambda a: np.asarray(a, dtype=np.float64)
    return lambda a: bf16(np.asarray(a, dtype=np.float32)).astype(np.float64)


def forward(prm, feats, exact: bool = False):
    """Logits [n, 65] and the activations as the kernels see them (BF16-rounded unless
    exact, which keeps everything in float64 for finite-difference checks)."""
    r = _rounder(exact)
    W1, b1, W2, b2, W3, b3 = (np.asarray(a, np.float64) for a in unpack(prm))
    n = feats.shape[0]
    X = np.zeros((n, NI))
    X[:, :NF] = feats
    X = r(X)
    W1b, W2b, W3b = r(W1), r(W2), r(W3)
    H1 = r(np.maximum(X @ W1b.T + b1, 0.0))
    H2 = r(np.maximum(H1 @ W2b.T + b2, 0.0))
    L = H2 @ W3b.T + b3
    return L[:, :NK + NW], (X, H1, H2, W1b, W2b, W3b, L)


def loss_and_grad(prm, feats, wlab, klab, scale, exact: bool = False):
    """scale * summed cross-entropy of both heads, and its gradient (float64)."""
    r = _rounder(exact)
    logits, (X, H1, H2, W1b, W2b, W3b, L) = forward(prm, feats, exact)
    n = feats.shape[0]
    D3 = np.zeros((n, NOP))
    loss = 0.0
    for lo, nn, lab in ((0, NK, np.asarray(klab, int)), (NK, NW, np.asarray(wlab, int))):
        z = L[:, lo:lo + nn] if exact else L[:, lo:lo + nn].astype(np.float32).astype(np.float64)
        m = z.max(axis=1, keepdims=True)
        lse = m[:, 0] + np.log(np.exp(z - m).sum(axis=1))
        loss += float((lse - z[np.arange(n), lab]).sum()) * scale
        p = np.exp(z - lse[:, None])
        p[np.arange(n), lab] -= 1.0
        D3[:, lo:lo + nn] = p * scale
    D3 = r(D3)
    g = np.zeros(NPARAM)
    gW3 = D3[:, :NO].T @ H2
    gb3 = D3[:, :NO].sum(axis=0)
    W3T = np.zeros((NH, NOP))
    W3T[:, :NO] = W3b.T
    D2 = r((D3 @ W3T.T) * (H2 > 0))
    gW2 = D2.T @ H1
    gb2 = D2.sum(axis=0)
    D1 = r((D2 @ W2b) * (H1 > 0))
    gW1 = D1.T @ X
    gb1 = D1.sum(axis=0)
    for name, val in (("W1", gW1), ("b1", gb1), ("W2", gW2), ("b2", gb2), ("W3", gW3), ("b3", gb3)):
        a, b = OFF[name]
        g[a:b] = val.ravel()
    return loss, g
