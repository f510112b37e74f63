// Zstandard frame decoder (RFC 8878) usable from host and device code, for the zstd level-3
// frames that wrap the containers (composer/utils.hpp:11-53 writes them with libzstd).
// Decoding is deterministic, so any correct decoder returns libzstd's bytes.
//
// Supported: single zstd frames without dictionary, raw / RLE / compressed blocks, raw / RLE /
// Huffman (1 or 4 streams, tree or repeated tree) literals, predefined / RLE / FSE / repeated
// sequence tables, repeat offsets, an optional content checksum (skipped, not verified).
//
// A Team is the set of threads that decode one frame together.  On the GPU it is a warp:
// every lane runs every step on the same data (the same branches; same-address loads are
// broadcasts), and only the stores are split: byte copies and Huffman table fills go
// lane-strided, the four Huffman literal streams go to lanes 0-3, FSE tables are built by
// lane 0, and a warp barrier separates each batch of stores from the reads that follow.
// Every branch depends only on values that all lanes hold alike, so the lanes never diverge
// around a barrier.  On the host a Team is one thread (SoloTeam).
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define ZD_HD __host__ __device__ __forceinline__
#else
#define ZD_HD inline
#endif

namespace xnyz {
namespace zd {

using u8 = uint8_t;
using u16 = uint16_t;
using u32 = uint32_t;
using u64 = unsigned long long;
using i64 = long long;

enum : int {
    kOk = 0,
    kErrFormat = -1,     // not a frame this decoder handles, or a corrupt one
    kErrDstSize = -2,    // output larger than the destination
    kErrTruncated = -3,  // input ends early
};

constexpr int kMaxBlock = 128 * 1024;
constexpr int kHufMaxBits = 11;

// Workspace of one decoder (global memory on the GPU: the literal buffer is 128 KB).
struct FseEntry {
    u16 base;  // next-state baseline
    u8 sym;
    u8 nb;     // bits to read
};
struct Workspace {
    u8 lit[kMaxBlock + 32];
    u16 huf[1 << kHufMaxBits];  // (symbol << 8) | bits
    FseEntry ll[512], of[256], ml[512];
};
// Table sizes of the frame so far, held by each thread of the team.
struct Logs {
    int huf_bits = 0;                      // 0: no Huffman table yet
    int ll = -1, of = -1, ml = -1;         // -1: no sequence table yet
};

// One host thread.
struct SoloTeam {
    int rank = 0;
    static constexpr int size = 1;
    void sync() const {}
    int min(int v) const { return v; }
    int bcast0(int v) const { return v; }
};

#ifdef __CUDACC__
// One warp (all 32 lanes active).  sync() puts a block-scope fence between two warp
// barriers: with the barrier alone, lanes still copying one block's last literals read
// bytes that another lane had already overwritten with the next block's literals (seen on
// sm_100a in one of the test frames); with the fence every lane's earlier loads and stores
// are performed before any lane goes on.
struct WarpTeam {
    int rank;
    static constexpr int size = 32;
    __device__ __forceinline__ void sync() const {
        __syncwarp();
        __threadfence_block();
        __syncwarp();
    }
    __device__ __forceinline__ int min(int v) const { return __reduce_min_sync(0xffffffffu, v); }
    __device__ __forceinline__ int bcast0(int v) const { return __shfl_sync(0xffffffffu, v, 0); }
};
#endif

// ---- little-endian reads ----
ZD_HD u32 rd16(const u8* p) { return (u32)p[0] | ((u32)p[1] << 8); }
ZD_HD u32 rd24(const u8* p) { return (u32)p[0] | ((u32)p[1] << 8) | ((u32)p[2] << 16); }
ZD_HD u32 rd32(const u8* p) { return rd16(p) | (rd16(p + 2) << 16); }
ZD_HD int highbit(u32 v) {
    int n = -1;
    while (v) {
        v >>= 1;
        ++n;
    }
    return n;
}

// Backward bit stream (FSE / Huffman payloads): bits are consumed from the end of the
// buffer towards its start; the last byte's highest set bit marks the end of the padding.
struct BackBits {
    const u8* buf;
    i64 len;    // bytes
    i64 pos;    // bits not yet consumed (from bit 0 of buf)
    i64 total;  // bits after the padding
    i64 wb;     // first byte of the cached 8-byte window
    u64 win;    // buf[wb .. wb+8), bytes outside the buffer as zero
    ZD_HD bool init(const u8* b, u64 n) {
        buf = b;
        len = (i64)n;
        wb = -(1ll << 40);
        if (!n || !b[n - 1]) return false;
        total = (i64)n * 8 - 8 + highbit(b[n - 1]);
        pos = total;
        return true;
    }
    // n <= 32 bits, most significant first; bits before the start read as zero
    ZD_HD u32 read(int n) {
        if (n == 0) return 0;
        pos -= n;
        return peek_at(pos, n);
    }
    ZD_HD u32 peek(int n) { return n ? peek_at(pos - n, n) : 0; }
    // The bits [p, p+n) need bytes p/8 .. p/8+4; the window is refilled 3 bytes below p/8,
    // so the reads that follow (towards the start) hit it for about 32 bits.
    ZD_HD u32 peek_at(i64 p, int n) {
        const i64 byte0 = p >> 3;  // arithmetic shift: negative positions round down
        if (byte0 < wb || byte0 > wb + 3) {
            wb = byte0 - 3;
            u64 v = 0;
            for (int k = 0; k < 8; ++k) {
                const i64 b = wb + k;
                const u64 x = (b >= 0 && b < len) ? buf[b] : 0;
                v |= x << (8 * k);
            }
            win = v;
        }
        const int sh = (int)(p - wb * 8);
        return (u32)((win >> sh) & ((1ull << n) - 1));
    }
    ZD_HD bool overflow() const { return pos < 0; }
};

// ---- FSE ----
// Reads a normalized distribution (RFC 8878 4.1.1); returns bytes used or < 0.
ZD_HD int read_ncount(const u8* src, u64 len, int max_log, int max_sym, short* norm, int& nsym, int& log) {
    if (len < 1) return kErrTruncated;
    i64 bitpos = 0;
    auto bits = [&](int n) -> u32 {
        u32 v = 0;
        for (int k = 0; k < n; ++k) {
            const i64 b = (bitpos + k) >> 3;
            const u32 bit = (b < (i64)len) ? (src[b] >> ((bitpos + k) & 7)) & 1u : 0u;
            v |= bit << k;
        }
        return v;
    };
    log = (int)bits(4) + 5;
    bitpos += 4;
    if (log > max_log) return kErrFormat;
    int remaining = (1 << log) + 1;
    int threshold = 1 << log;
    int nb = log + 1;
    int s = 0;
    bool prev0 = false;
    while (remaining > 1 && s <= max_sym) {
        if (prev0) {
            // repeat flags: 2 bits each, 3 means "3 more and another flag"
            int n0 = s;
            for (;;) {
                const u32 f = bits(2);
                bitpos += 2;
                n0 += (int)f;
                if (f != 3) break;
            }
            if (n0 > max_sym + 1) return kErrFormat;
            while (s < n0) norm[s++] = 0;
            if (s > max_sym) break;
        }
        const int max = (2 * threshold - 1) - remaining;
        int count;
        const u32 low = bits(nb - 1);
        if ((int)low < max) {
            count = (int)low;
            bitpos += nb - 1;
        } else {
            u32 v = bits(nb);
            if ((int)v >= threshold) v -= max;
            count = (int)v;
            bitpos += nb;
        }
        count--;  // -1: "less than 1"
        remaining -= count < 0 ? -count : count;
        norm[s++] = (short)count;
        prev0 = count == 0;
        while (remaining < threshold) {
            nb--;
            threshold >>= 1;
        }
    }
    if (remaining != 1 || s > max_sym + 1) return kErrFormat;
    nsym = s;
    for (int k = s; k <= max_sym; ++k) norm[k] = 0;
    if (bitpos > (i64)len * 8) return kErrTruncated;
    return (int)((bitpos + 7) >> 3);
}

// Decoding table from a normalized distribution (RFC 8878 4.1.1).
ZD_HD int build_fse(const short* norm, int nsym, int log, FseEntry* t) {
    const int size = 1 << log;
    int high = size - 1;
    u16 next[256];
    for (int s = 0; s < nsym; ++s) {
        if (norm[s] == -1) {
            t[high--].sym = (u8)s;
            next[s] = 1;
        } else {
            next[s] = (u16)norm[s];
        }
    }
    const int step = (size >> 1) + (size >> 3) + 3, mask = size - 1;
    int p = 0;
    for (int s = 0; s < nsym; ++s) {
        for (int i = 0; i < norm[s]; ++i) {
            t[p].sym = (u8)s;
            do {
                p = (p + step) & mask;
            } while (p > high);
        }
    }
    if (p != 0) return kErrFormat;
    for (int i = 0; i < size; ++i) {
        const int s = t[i].sym;
        const u32 ns = next[s]++;
        const int nb = log - highbit(ns);
        t[i].nb = (u8)nb;
        t[i].base = (u16)((ns << nb) - size);
    }
    return kOk;
}

ZD_HD void rle_fse(FseEntry* t, u8 sym) {
    t[0].sym = sym;
    t[0].nb = 0;
    t[0].base = 0;
}

// Predefined distributions (RFC 8878 3.1.1.3.2.2).
ZD_HD void default_ll(short* n) {
    const short d[36] = {4, 3, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 1, 1, 1, 2, 2,
                         2, 2, 2, 2, 2, 2, 2, 3, 2, 1, 1, 1, 1, 1, -1, -1, -1, -1};
    for (int i = 0; i < 36; ++i) n[i] = d[i];
}
ZD_HD void default_ml(short* n) {
    const short d[53] = {1, 4, 3, 2, 2, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1,
                         1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1, -1, -1};
    for (int i = 0; i < 53; ++i) n[i] = d[i];
}
ZD_HD void default_of(short* n) {
    const short d[29] = {1, 1, 1, 1, 1, 1, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1};
    for (int i = 0; i < 29; ++i) n[i] = d[i];
}

// Literal / match length codes: baseline and extra bits (RFC 8878 3.1.1.3.2.1.1).
ZD_HD void ll_code(int c, u32& base, int& bits) {
    const u32 b[36] = {0,  1,  2,  3,  4,  5,  6,  7,  8,   9,   10,  11,   12,   13,   14,   15,    16,    18,
                       20, 22, 24, 28, 32, 40, 48, 64, 128, 256, 512, 1024, 2048, 4096, 8192, 16384, 32768, 65536};
    const u8 n[36] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 3, 3, 4, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16};
    base = b[c];
    bits = n[c];
}
ZD_HD void ml_code(int c, u32& base, int& bits) {
    if (c < 32) {
        base = (u32)c + 3;
        bits = 0;
        return;
    }
    const u32 b[21] = {35, 37, 39, 41, 43, 47, 51, 59, 67, 83, 99, 131, 259, 515, 1027, 2051, 4099, 8195, 16387, 32771, 65539};
    const u8 n[21] = {1, 1, 1, 1, 2, 2, 3, 3, 4, 4, 5, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16};
    base = b[c - 32];
    bits = n[c - 32];
}

// ---- Huffman literals ----
// Tree description (RFC 8878 4.2.1) -> ws.huf; returns bytes used or < 0.
template <class Team>
ZD_HD int read_huf_tree(const u8* src, u64 len, Workspace& ws, int& huf_bits, const Team& team) {
    if (len < 1) return kErrTruncated;
    u8 w[256];
    int nw = 0;
    const u32 hb = src[0];
    u64 used;
    if (hb < 128) {  // FSE-compressed weights, two interleaved states
        if (1 + hb > len) return kErrTruncated;
        short norm[256];
        int nsym = 0, log = 0;
        const int r = read_ncount(src + 1, hb, 6, 255, norm, nsym, log);
        if (r < 0) return r;
        FseEntry t[64];
        if (build_fse(norm, nsym, log, t) != kOk) return kErrFormat;
        BackBits bb;
        if (!bb.init(src + 1 + r, hb - (u64)r)) return kErrFormat;
        u32 s1 = bb.read(log), s2 = bb.read(log);
        for (;;) {
            if (nw >= 255) return kErrFormat;
            w[nw++] = t[s1].sym;
            s1 = t[s1].base + bb.read(t[s1].nb);
            if (bb.overflow()) {
                w[nw++] = t[s2].sym;
                break;
            }
            if (nw >= 255) return kErrFormat;
            w[nw++] = t[s2].sym;
            s2 = t[s2].base + bb.read(t[s2].nb);
            if (bb.overflow()) {
                w[nw++] = t[s1].sym;
                break;
            }
        }
        used = 1 + hb;
    } else {  // direct 4-bit weights
        nw = (int)hb - 127;
        const u64 nb = ((u64)nw + 1) / 2;
        if (1 + nb > len) return kErrTruncated;
        for (int i = 0; i < nw; ++i) w[i] = (u8)((i & 1) ? (src[1 + i / 2] & 15) : (src[1 + i / 2] >> 4));
        used = 1 + nb;
    }
    // the last weight completes the sum to a power of two
    u32 sum = 0;
    for (int i = 0; i < nw; ++i) {
        if (w[i] > kHufMaxBits + 1) return kErrFormat;
        if (w[i]) sum += 1u << (w[i] - 1);
    }
    if (!sum) return kErrFormat;
    const int maxb = highbit(sum) + 1;
    if (maxb > kHufMaxBits) return kErrFormat;
    const u32 rest = (1u << maxb) - sum;
    if (rest & (rest - 1)) return kErrFormat;
    if (nw > 255) return kErrFormat;  // 255 explicit weights at most: the implied one is the 256th
    w[nw++] = (u8)(highbit(rest) + 1);
    // codes in order of increasing weight, then symbol; weight w spans 2^(w-1) entries
    u32 start[kHufMaxBits + 2] = {};
    u32 cnt[kHufMaxBits + 2] = {};
    for (int i = 0; i < nw; ++i) cnt[w[i]]++;
    u32 acc = 0;
    for (int k = 1; k <= maxb; ++k) {
        start[k] = acc;
        acc += cnt[k] << (k - 1);
    }
    for (int s = 0; s < nw; ++s) {
        const int k = w[s];
        if (!k) continue;
        const u32 span = 1u << (k - 1);
        const u16 e = (u16)((s << 8) | (maxb + 1 - k));
        for (u32 j = team.rank; j < span; j += team.size) ws.huf[start[k] + j] = e;
        start[k] += span;
    }
    huf_bits = maxb;
    team.sync();
    return (int)used;
}

// Decodes n literals; stores out[i] only where (i & wmask) == wrank.
ZD_HD int huf_stream(const u8* src, u64 len, u8* out, u64 n, const Workspace& ws, int mb, u64 wmask, u64 wrank) {
    BackBits bb;
    if (!bb.init(src, len)) return kErrFormat;
    for (u64 i = 0; i < n; ++i) {
        const u16 e = ws.huf[bb.peek(mb)];
        if ((i & wmask) == wrank) out[i] = (u8)(e >> 8);
        bb.pos -= (e & 0xff);
    }
    if (bb.pos != 0) return kErrFormat;
    return kOk;
}

// Literals section; returns bytes used or < 0, *nlit = regenerated size.
// The literals are in ws.lit for every lane when it returns.
template <class Team>
ZD_HD int read_literals(const u8* src, u64 len, Workspace& ws, int& huf_bits, u64& nlit, const Team& team) {
    team.sync();  // every lane is done with the previous block's literals
    if (len < 1) return kErrTruncated;
    const int type = src[0] & 3, fmt = (src[0] >> 2) & 3;
    if (type < 2) {
        u64 h, n;
        if (fmt == 0 || fmt == 2) {
            h = 1;
            n = src[0] >> 3;
        } else if (fmt == 1) {
            if (len < 2) return kErrTruncated;
            h = 2;
            n = (src[0] >> 4) | ((u32)src[1] << 4);
        } else {
            if (len < 3) return kErrTruncated;
            h = 3;
            n = (src[0] >> 4) | ((u32)src[1] << 4) | ((u32)src[2] << 12);
        }
        if (n > kMaxBlock) return kErrFormat;
        if (type == 0) {
            if (h + n > len) return kErrTruncated;
            for (u64 i = team.rank; i < n; i += team.size) ws.lit[i] = src[h + i];
            team.sync();
            nlit = n;
            return (int)(h + n);
        }
        if (h + 1 > len) return kErrTruncated;
        for (u64 i = team.rank; i < n; i += team.size) ws.lit[i] = src[h];
        team.sync();
        nlit = n;
        return (int)(h + 1);
    }
    u64 h, regen, comp;
    int streams = fmt == 0 ? 1 : 4;
    if (fmt < 2) {
        if (len < 3) return kErrTruncated;
        const u32 v = rd24(src);
        h = 3;
        regen = (v >> 4) & 0x3ff;
        comp = (v >> 14) & 0x3ff;
    } else if (fmt == 2) {
        if (len < 4) return kErrTruncated;
        const u32 v = rd32(src);
        h = 4;
        regen = (v >> 4) & 0x3fff;
        comp = (v >> 18) & 0x3fff;
    } else {
        if (len < 5) return kErrTruncated;
        const u64 v = (u64)rd32(src) | ((u64)src[4] << 32);
        h = 5;
        regen = (v >> 4) & 0x3ffff;
        comp = (v >> 22) & 0x3ffff;
    }
    if (regen > kMaxBlock || h + comp > len) return kErrFormat;
    const u8* p = src + h;
    u64 rem = comp;
    if (type == 2) {
        const int r = read_huf_tree(p, rem, ws, huf_bits, team);
        if (r < 0) return r;
        p += r;
        rem -= (u64)r;
    } else if (!huf_bits) {
        return kErrFormat;  // repeated tree without a previous one
    }
    if (streams == 1) {
        const int r = huf_stream(p, rem, ws.lit, regen, ws, huf_bits, (u64)team.size - 1, (u64)team.rank);
        team.sync();
        if (r < 0) return r;
    } else {
        if (rem < 6) return kErrTruncated;
        const u64 s1 = rd16(p), s2 = rd16(p + 2), s3 = rd16(p + 4);
        if (6 + s1 + s2 + s3 > rem) return kErrTruncated;
        const u64 s4 = rem - 6 - s1 - s2 - s3;
        const u64 seg = (regen + 3) / 4;
        if (3 * seg > regen) return kErrFormat;
        const u64 sz[4] = {s1, s2, s3, s4};
        // a one-thread team decodes the four streams in turn; a warp gives stream k to the
        // lanes k, k+4, ... of which lane k stores
        const int first = team.size == 1 ? 0 : (team.rank & 3);
        const int step = team.size == 1 ? 1 : 4;
        const u64 wrank = team.rank < 4 ? 0 : 1;
        int worst = kOk;
        for (int k = first; k < 4; k += step) {
            u64 start = 6;
            for (int j = 0; j < k; ++j) start += sz[j];
            const u64 cnt = k < 3 ? seg : regen - 3 * seg;
            const int r = huf_stream(p + start, sz[k], ws.lit + (u64)k * seg, cnt, ws, huf_bits, 0, wrank);
            if (r < worst) worst = r;
        }
        worst = team.min(worst);
        team.sync();
        if (worst < 0) return worst;
    }
    nlit = regen;
    return (int)(h + comp);
}

// Sequence table for one of LL / OF / ML by its mode; returns bytes used or < 0.
// The table is built by rank 0; every lane sees it when this returns.
template <class Team>
ZD_HD int read_table(int mode, const u8* src, u64 len, FseEntry* t, int& log, int max_log, int max_sym,
                     int which, const Team& team) {
    if (mode == 0) {
        short norm[64];
        if (which == 0) default_ll(norm);
        else if (which == 1) default_of(norm);
        else default_ml(norm);
        const int nsym = which == 0 ? 36 : which == 1 ? 29 : 53;
        log = which == 1 ? 5 : 6;
        int rc = kOk;
        if (team.rank == 0) rc = build_fse(norm, nsym, log, t);
        rc = team.bcast0(rc);
        team.sync();
        return rc == kOk ? 0 : kErrFormat;
    }
    if (mode == 1) {
        if (len < 1) return kErrTruncated;
        if (src[0] > max_sym) return kErrFormat;
        if (team.rank == 0) rle_fse(t, src[0]);
        team.sync();
        log = 0;
        return 1;
    }
    if (mode == 2) {
        short norm[64];
        int nsym = 0;
        const int r = read_ncount(src, len, max_log, max_sym, norm, nsym, log);
        if (r < 0) return r;
        int rc = kOk;
        if (team.rank == 0) rc = build_fse(norm, nsym, log, t);
        rc = team.bcast0(rc);
        team.sync();
        if (rc != kOk) return kErrFormat;
        return r;
    }
    return log < 0 ? kErrFormat : 0;  // repeat the previous table
}

// One compressed block into dst[op ...]; returns bytes written or < 0.
template <class Team>
ZD_HD i64 decode_block(const u8* src, u64 len, u8* dst, u64 op, u64 cap, Workspace& ws, Logs& lg, u32* rep,
                       const Team& team) {
    u64 nlit = 0;
    const int lr = read_literals(src, len, ws, lg.huf_bits, nlit, team);
    if (lr < 0) return lr;
    const u8* p = src + lr;
    u64 rem = len - (u64)lr;
    if (rem < 1) return kErrTruncated;
    u64 nseq;
    if (p[0] == 0) {
        nseq = 0;
        p += 1;
        rem -= 1;
    } else if (p[0] < 128) {
        nseq = p[0];
        p += 1;
        rem -= 1;
    } else if (p[0] < 255) {
        if (rem < 2) return kErrTruncated;
        nseq = ((u64)(p[0] - 128) << 8) + p[1];
        p += 2;
        rem -= 2;
    } else {
        if (rem < 3) return kErrTruncated;
        nseq = (u64)p[1] + ((u64)p[2] << 8) + 0x7f00;
        p += 3;
        rem -= 3;
    }
    u64 o = op;
    if (nseq == 0) {
        if (o + nlit > cap) return kErrDstSize;
        for (u64 i = team.rank; i < nlit; i += team.size) dst[o + i] = ws.lit[i];
        return (i64)nlit;
    }
    if (rem < 1) return kErrTruncated;
    const int modes = p[0];
    p += 1;
    rem -= 1;
    int r = read_table(modes >> 6, p, rem, ws.ll, lg.ll, 9, 35, 0, team);
    if (r < 0) return r;
    p += r;
    rem -= (u64)r;
    r = read_table((modes >> 4) & 3, p, rem, ws.of, lg.of, 8, 31, 1, team);
    if (r < 0) return r;
    p += r;
    rem -= (u64)r;
    r = read_table((modes >> 2) & 3, p, rem, ws.ml, lg.ml, 9, 52, 2, team);
    if (r < 0) return r;
    p += r;
    rem -= (u64)r;
    BackBits bb;
    if (!bb.init(p, rem)) return kErrFormat;
    u32 sll = bb.read(lg.ll), sof = bb.read(lg.of), sml = bb.read(lg.ml);
    u64 li = 0;
    u64 synced = o;  // every lane sees the output below this position
    for (u64 k = 0; k < nseq; ++k) {
        const int llc = ws.ll[sll].sym, ofc = ws.of[sof].sym, mlc = ws.ml[sml].sym;
        if (ofc > 31) return kErrFormat;
        const u32 ofv = (1u << ofc) + bb.read(ofc);
        u32 mb, lb;
        int mn, ln;
        ml_code(mlc, mb, mn);
        ll_code(llc, lb, ln);
        const u32 ml = mb + bb.read(mn);
        const u32 ll = lb + bb.read(ln);
        u32 off;
        if (ofv > 3) {
            off = ofv - 3;
            rep[2] = rep[1];
            rep[1] = rep[0];
            rep[0] = off;
        } else {
            const u32 idx = ofv + (ll == 0 ? 1u : 0u);
            if (idx == 1) {
                off = rep[0];
            } else if (idx == 2) {
                off = rep[1];
                rep[1] = rep[0];
                rep[0] = off;
            } else if (idx == 3) {
                off = rep[2];
                rep[2] = rep[1];
                rep[1] = rep[0];
                rep[0] = off;
            } else {
                off = rep[0] - 1;
                if (off == 0) return kErrFormat;
                rep[2] = rep[1];
                rep[1] = rep[0];
                rep[0] = off;
            }
        }
        if (k + 1 < nseq) {  // state updates: literal length, match length, offset
            sll = ws.ll[sll].base + bb.read(ws.ll[sll].nb);
            sml = ws.ml[sml].base + bb.read(ws.ml[sml].nb);
            sof = ws.of[sof].base + bb.read(ws.of[sof].nb);
        }
        if (li + ll > nlit || o + ll + ml > cap) return li + ll > nlit ? kErrFormat : kErrDstSize;
        for (u32 i = team.rank; i < ll; i += team.size) dst[o + i] = ws.lit[li + i];
        o += ll;
        li += ll;
        if (off > o) return kErrFormat;
        // Byte i of the match repeats byte i mod off of the off bytes before it, all written
        // before this match: the lanes copy in any order once those bytes are visible, which
        // needs a barrier only when the sources reach past the last one.
        const u64 from = o - off;
        if (from + (off < ml ? off : ml) > synced) {
            team.sync();
            synced = o;
        }
        if (off >= ml) {
            for (u32 i = team.rank; i < ml; i += team.size) dst[o + i] = dst[from + i];
        } else {
            for (u32 i = team.rank; i < ml; i += team.size) dst[o + i] = dst[from + i % off];
        }
        o += ml;
    }
    if (bb.pos != 0) return kErrFormat;
    if (o + (nlit - li) > cap) return kErrDstSize;
    for (u64 i = li + team.rank; i < nlit; i += team.size) dst[o + (i - li)] = ws.lit[i];
    o += nlit - li;
    return (i64)(o - op);
}

// One frame: src[0..len) -> dst[0..cap); returns the content size or < 0.
template <class Team>
ZD_HD i64 decode_frame(const u8* src, u64 len, u8* dst, u64 cap, Workspace& ws, const Team& team) {
    if (len < 6 || rd32(src) != 0xFD2FB528u) return kErrFormat;
    const u32 fhd = src[4];
    const int fcs_flag = fhd >> 6, single = (fhd >> 5) & 1, checksum = (fhd >> 2) & 1, did = fhd & 3;
    if (fhd & 8) return kErrFormat;  // reserved bit
    u64 p = 5;
    if (!single) p += 1;  // window descriptor
    const int did_bytes = did == 0 ? 0 : did == 1 ? 1 : did == 2 ? 2 : 4;
    if (did_bytes) return kErrFormat;  // dictionaries are not used by the container frames
    const int fcs_bytes = fcs_flag == 0 ? (single ? 1 : 0) : fcs_flag == 1 ? 2 : fcs_flag == 2 ? 4 : 8;
    if (p + fcs_bytes > len) return kErrTruncated;
    u64 fcs = ~0ull;
    if (fcs_bytes == 1) fcs = src[p];
    else if (fcs_bytes == 2) fcs = rd16(src + p) + 256;
    else if (fcs_bytes == 4) fcs = rd32(src + p);
    else if (fcs_bytes == 8) fcs = (u64)rd32(src + p) | ((u64)rd32(src + p + 4) << 32);
    p += fcs_bytes;
    Logs lg;
    u32 rep[3] = {1, 4, 8};
    u64 o = 0;
    for (;;) {
        if (p + 3 > len) return kErrTruncated;
        const u32 bh = rd24(src + p);
        p += 3;
        const int last = bh & 1, type = (bh >> 1) & 3;
        const u64 bsize = bh >> 3;
        if (type == 3) return kErrFormat;
        if (type == 0) {
            if (p + bsize > len) return kErrTruncated;
            if (o + bsize > cap) return kErrDstSize;
            for (u64 i = team.rank; i < bsize; i += team.size) dst[o + i] = src[p + i];
            o += bsize;
            p += bsize;
        } else if (type == 1) {
            if (p + 1 > len) return kErrTruncated;
            if (o + bsize > cap) return kErrDstSize;
            for (u64 i = team.rank; i < bsize; i += team.size) dst[o + i] = src[p];
            o += bsize;
            p += 1;
        } else {
            if (bsize > kMaxBlock || p + bsize > len) return kErrTruncated;
            const i64 w = decode_block(src + p, bsize, dst, o, cap, ws, lg, rep, team);
            if (w < 0) return w;
            o += (u64)w;
            p += bsize;
        }
        if (last) break;
    }
    if (checksum) p += 4;
    if (p > len) return kErrTruncated;
    if (fcs != ~0ull && fcs != o) return kErrFormat;
    return (i64)o;
}

}  // namespace zd
}  // namespace xnyz
