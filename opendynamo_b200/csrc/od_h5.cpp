// Solver-native state files: the HDF5 subset the reference writes and reads
// (src/io.rs:59-234), implemented from the public HDF5 file-format
// specification (no libhdf5 in this environment).
//
// File layout written (the "earliest" format libhdf5 uses by default):
//   superblock v0, object headers v1, old-style groups (symbol table message,
//   local heap, v1 B-tree, symbol table nodes);
//   root attributes nx ny nz fr_order step (u64), t lx ly lz (f64),
//   u_real (3-byte fixed ASCII); group /data with 1-D datasets
//   rho rhou rhov rhow E of f32 or f64 (io.rs:94-134);
//   compression (io.rs:17-52, config.rs:182-203): "none" contiguous;
//   "gzipN" chunked (262144 elements) with shuffle + deflate N; "blosc-lz4" /
//   "blosc-zstd" chunked with the Blosc filter (id 32001, byte shuffle,
//   clevel 9 / 5 as io.rs:38-39).
// Reader: the same subset, plus what libhdf5 adds to files it writes —
// object-header continuation blocks, multi-level chunk B-trees, full-size
// B-tree and symbol-table nodes, any message order; it validates mesh,
// fr_order and u_real like io.rs:163-234 and reads f64 planes as f64 (the
// reference reads every plane as f32, io.rs:221, which makes its f64 resume
// inexact).

#include <dlfcn.h>
#include <zlib.h>

#include "opendynamo.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace {

constexpr uint64_t UNDEF = ~0ull;
constexpr size_t CHUNK_ELEMS = 1u << 18;  // io.rs:11
constexpr size_t kEncodeThreads = 4;      // the reference's blosc thread count (solver.rs:213-220)
const char* const VAR_NAMES[5] = {"rho", "rhou", "rhov", "rhow", "E"};

struct H5Error : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// ---------------------------------------------------------------- bytes
struct Buf {
    std::vector<uint8_t> b;
    void u8(uint8_t v) { b.push_back(v); }
    void u16(uint16_t v) { for (int i = 0; i < 2; ++i) b.push_back((uint8_t)(v >> (8 * i))); }
    void u32(uint32_t v) { for (int i = 0; i < 4; ++i) b.push_back((uint8_t)(v >> (8 * i))); }
    void u64(uint64_t v) { for (int i = 0; i < 8; ++i) b.push_back((uint8_t)(v >> (8 * i))); }
    void raw(const void* p, size_t n) { b.insert(b.end(), (const uint8_t*)p, (const uint8_t*)p + n); }
    void zeros(size_t n) { b.insert(b.end(), n, 0); }
    void pad8() { while (b.size() % 8) b.push_back(0); }
    size_t size() const { return b.size(); }
    void put64(size_t at, uint64_t v) { for (int i = 0; i < 8; ++i) b[at + i] = (uint8_t)(v >> (8 * i)); }
    void put32(size_t at, uint32_t v) { for (int i = 0; i < 4; ++i) b[at + i] = (uint8_t)(v >> (8 * i)); }
};

uint64_t rd(const uint8_t* p, int n) {
    uint64_t v = 0;
    for (int i = 0; i < n; ++i) v |= (uint64_t)p[i] << (8 * i);
    return v;
}

// ---------------------------------------------------------------- codecs
struct Lz4Zstd {
    void* lz4 = nullptr;
    void* zstd = nullptr;
    int (*lz4_compress)(const char*, char*, int, int) = nullptr;
    int (*lz4_bound)(int) = nullptr;
    int (*lz4_decompress)(const char*, char*, int, int) = nullptr;
    size_t (*zstd_compress)(void*, size_t, const void*, size_t, int) = nullptr;
    size_t (*zstd_bound)(size_t) = nullptr;
    size_t (*zstd_decompress)(void*, size_t, const void*, size_t) = nullptr;
    unsigned (*zstd_iserror)(size_t) = nullptr;
    Lz4Zstd() {
        lz4 = dlopen("liblz4.so.1", RTLD_NOW | RTLD_LOCAL);
        if (lz4) {
            lz4_compress = (decltype(lz4_compress))dlsym(lz4, "LZ4_compress_default");
            lz4_bound = (decltype(lz4_bound))dlsym(lz4, "LZ4_compressBound");
            lz4_decompress = (decltype(lz4_decompress))dlsym(lz4, "LZ4_decompress_safe");
        }
        zstd = dlopen("libzstd.so.1", RTLD_NOW | RTLD_LOCAL);
        if (zstd) {
            zstd_compress = (decltype(zstd_compress))dlsym(zstd, "ZSTD_compress");
            zstd_bound = (decltype(zstd_bound))dlsym(zstd, "ZSTD_compressBound");
            zstd_decompress = (decltype(zstd_decompress))dlsym(zstd, "ZSTD_decompress");
            zstd_iserror = (decltype(zstd_iserror))dlsym(zstd, "ZSTD_isError");
        }
    }
};

Lz4Zstd& codecs() {
    static Lz4Zstd c;
    return c;
}

void shuffle(const uint8_t* in, uint8_t* out, size_t n, size_t ts) {
    const size_t ne = n / ts;
    for (size_t i = 0; i < ne; ++i)
        for (size_t b = 0; b < ts; ++b) out[b * ne + i] = in[i * ts + b];
    std::memcpy(out + ne * ts, in + ne * ts, n - ne * ts);
}

void unshuffle(const uint8_t* in, uint8_t* out, size_t n, size_t ts) {
    const size_t ne = n / ts;
    for (size_t i = 0; i < ne; ++i)
        for (size_t b = 0; b < ts; ++b) out[i * ts + b] = in[b * ne + i];
    std::memcpy(out + ne * ts, in + ne * ts, n - ne * ts);
}

std::vector<uint8_t> deflate_bytes(const std::vector<uint8_t>& in, int level) {
    uLongf cap = compressBound((uLong)in.size());
    std::vector<uint8_t> out(cap);
    if (compress2(out.data(), &cap, in.data(), (uLong)in.size(), level) != Z_OK) throw H5Error("deflate failed");
    out.resize(cap);
    return out;
}

std::vector<uint8_t> inflate_bytes(const uint8_t* in, size_t n, size_t expect) {
    std::vector<uint8_t> out(expect);
    uLongf len = (uLongf)expect;
    int rc = uncompress(out.data(), &len, in, (uLong)n);
    if (rc != Z_OK) throw H5Error("corrupt deflate chunk");
    out.resize(len);
    return out;
}

// Blosc (c-blosc 1.x frame): 16-byte header — version, versionlz, flags
// (0x1 byte shuffle, 0x2 stored, 0x4 bit shuffle, 0x10 blocks not split
// into per-byte streams, compressor format in bits 5-7: 0 blosclz, 1 lz4,
// 2 snappy, 3 zlib, 4 zstd), typesize, nbytes, blocksize, ctbytes; then one
// int32 start offset per block; each block is one stream, or typesize
// streams (one per byte of the shuffled type) when split, each stored as
// (int32 csize, bytes) and raw when csize equals the stream length.
std::vector<uint8_t> blosc_encode(const std::vector<uint8_t>& in, int typesize, bool zstd_codec, int clevel) {
    Lz4Zstd& c = codecs();
    if (zstd_codec ? !c.zstd_compress : !c.lz4_compress) throw H5Error("blosc codec library not available");
    const size_t nbytes = in.size();
    const size_t blocksize = std::min<size_t>(nbytes, 256 * 1024);
    const size_t nblocks = blocksize ? (nbytes + blocksize - 1) / blocksize : 0;
    Buf out;
    out.u8(2);                 // frame version
    out.u8(1);                 // codec format version
    out.u8((uint8_t)(0x1 | 0x10 | ((zstd_codec ? 4 : 1) << 5)));  // shuffled, one stream per block
    out.u8((uint8_t)typesize);
    out.u32((uint32_t)nbytes);
    out.u32((uint32_t)blocksize);
    out.u32(0);  // ctbytes, patched
    const size_t bstarts = out.size();
    out.zeros(4 * nblocks);
    std::vector<uint8_t> sh(blocksize), comp;
    for (size_t bi = 0; bi < nblocks; ++bi) {
        const size_t off = bi * blocksize;
        const size_t bs = std::min(blocksize, nbytes - off);
        out.put32(bstarts + 4 * bi, (uint32_t)out.size());
        shuffle(in.data() + off, sh.data(), bs, (size_t)typesize);
        size_t cs;
        if (zstd_codec) {
            comp.resize(c.zstd_bound(bs));
            cs = c.zstd_compress(comp.data(), comp.size(), sh.data(), bs, clevel);
            if (c.zstd_iserror(cs)) cs = bs + 1;
        } else {
            comp.resize((size_t)c.lz4_bound((int)bs));
            int r = c.lz4_compress((const char*)sh.data(), (char*)comp.data(), (int)bs, (int)comp.size());
            cs = r > 0 ? (size_t)r : bs + 1;
        }
        if (cs >= bs) {  // incompressible stream: stored raw
            out.u32((uint32_t)bs);
            out.raw(sh.data(), bs);
        } else {
            out.u32((uint32_t)cs);
            out.raw(comp.data(), cs);
        }
    }
    out.put32(12, (uint32_t)out.size());
    return out.b;
}

std::vector<uint8_t> blosc_decode(const uint8_t* in, size_t n) {
    if (n < 16) throw H5Error("corrupt blosc chunk");
    const uint8_t flags = in[2];
    const size_t typesize = in[3];
    const size_t nbytes = rd(in + 4, 4), blocksize = rd(in + 8, 4), ctbytes = rd(in + 12, 4);
    if (ctbytes > n || typesize == 0) throw H5Error("corrupt blosc chunk");
    std::vector<uint8_t> out(nbytes);
    if (flags & 0x2) {
        if (16 + nbytes > n) throw H5Error("corrupt blosc chunk");
        std::memcpy(out.data(), in + 16, nbytes);
        return out;
    }
    if (flags & 0x4) throw H5Error("blosc bit shuffle is not supported");
    const int codec = flags >> 5;
    Lz4Zstd& c = codecs();
    const size_t nblocks = blocksize ? (nbytes + blocksize - 1) / blocksize : 0;
    std::vector<uint8_t> tmp(blocksize);
    for (size_t bi = 0; bi < nblocks; ++bi) {
        const size_t off = bi * blocksize;
        const size_t bs = std::min(blocksize, nbytes - off);
        const bool leftover = bs < blocksize;
        const bool split = !(flags & 0x10) && !leftover && typesize <= 16 && blocksize / typesize >= 128;
        const size_t nstreams = split ? typesize : 1;
        const size_t neb = bs / nstreams;
        size_t pos = rd(in + 16 + 4 * bi, 4);
        for (size_t s = 0; s < nstreams; ++s) {
            if (pos + 4 > n) throw H5Error("corrupt blosc chunk");
            const size_t cs = rd(in + pos, 4);
            pos += 4;
            if (pos + cs > n) throw H5Error("corrupt blosc chunk");
            uint8_t* dst = tmp.data() + s * neb;
            if (cs == neb) {
                std::memcpy(dst, in + pos, neb);
            } else if (codec == 1) {
                if (!c.lz4_decompress) throw H5Error("liblz4 not available");
                if (c.lz4_decompress((const char*)in + pos, (char*)dst, (int)cs, (int)neb) != (int)neb)
                    throw H5Error("corrupt lz4 stream");
            } else if (codec == 4) {
                if (!c.zstd_decompress) throw H5Error("libzstd not available");
                if (c.zstd_decompress(dst, neb, in + pos, cs) != neb) throw H5Error("corrupt zstd stream");
            } else if (codec == 3) {
                uLongf len = (uLongf)neb;
                if (uncompress(dst, &len, in + pos, (uLong)cs) != Z_OK || len != neb)
                    throw H5Error("corrupt zlib stream");
            } else {
                throw H5Error("unsupported blosc codec");
            }
            pos += cs;
        }
        if (flags & 0x1)
            unshuffle(tmp.data(), out.data() + off, bs, typesize);
        else
            std::memcpy(out.data() + off, tmp.data(), bs);
    }
    return out;
}

// ---------------------------------------------------------------- writer
enum class Comp { None, Gzip, BloscLz4, BloscZstd };

struct Compression {
    Comp kind = Comp::None;
    int level = 0;
};

Compression parse_compression(const char* s) {
    std::string v = s ? s : "none";
    if (v == "none") return {Comp::None, 0};
    if (v == "blosc-lz4") return {Comp::BloscLz4, 9};   // io.rs:38
    if (v == "blosc-zstd") return {Comp::BloscZstd, 5}; // io.rs:39
    if (v.size() == 5 && v.compare(0, 4, "gzip") == 0 && v[4] >= '1' && v[4] <= '9') return {Comp::Gzip, v[4] - '0'};
    throw H5Error("invalid compression '" + v + "': expected \"none\", \"gzip1\"..\"gzip9\", \"blosc-lz4\" or \"blosc-zstd\"");
}

void dtype_float(Buf& m, int es) {
    m.u8(0x11);
    m.u8(0x20);
    m.u8(es == 4 ? 31 : 63);
    m.u8(0);
    m.u32((uint32_t)es);
    m.u16(0);
    m.u16((uint16_t)(8 * es));
    m.u8(es == 4 ? 23 : 52);
    m.u8(es == 4 ? 8 : 11);
    m.u8(0);
    m.u8(es == 4 ? 23 : 52);
    m.u32(es == 4 ? 127 : 1023);
}

void dtype_u64(Buf& m) {
    m.u8(0x10);
    m.u8(0);
    m.u8(0);
    m.u8(0);
    m.u32(8);
    m.u16(0);
    m.u16(64);
}

void dtype_str3(Buf& m) {
    m.u8(0x13);
    m.u8(0x01);  // null-padded, ASCII
    m.u8(0);
    m.u8(0);
    m.u32(3);
}

void message(Buf& oh, int& count, uint16_t type, const Buf& data, uint8_t flags = 0) {
    Buf d = data;
    d.pad8();
    oh.u16(type);
    oh.u16((uint16_t)d.size());
    oh.u8(flags);
    oh.zeros(3);
    oh.raw(d.b.data(), d.size());
    ++count;
}

Buf attribute(const char* name, void (*dtype)(Buf&), const void* value, size_t vsize) {
    Buf dt, ds, m;
    dtype(dt);
    ds.u8(1);
    ds.u8(0);  // scalar
    ds.u8(0);
    ds.u8(0);
    ds.u32(0);
    const size_t nlen = std::strlen(name) + 1;
    m.u8(1);
    m.u8(0);
    m.u16((uint16_t)nlen);
    m.u16((uint16_t)dt.size());
    m.u16((uint16_t)ds.size());
    m.raw(name, nlen);
    m.pad8();
    m.raw(dt.b.data(), dt.size());
    m.pad8();
    m.raw(ds.b.data(), ds.size());
    m.pad8();
    m.raw(value, vsize);
    return m;
}

Buf object_header(const std::vector<std::pair<uint16_t, Buf>>& msgs) {
    Buf body;
    int count = 0;
    for (auto& mm : msgs) message(body, count, mm.first, mm.second);
    Buf oh;
    oh.u8(1);
    oh.u8(0);
    oh.u16((uint16_t)count);
    oh.u32(1);
    oh.u32((uint32_t)body.size());
    oh.zeros(4);
    oh.raw(body.b.data(), body.size());
    return oh;
}

// local heap with the names at 8-byte aligned offsets ("" at 0)
struct Heap {
    Buf data;
    std::map<std::string, uint64_t> off;
    Heap() {
        data.zeros(8);
        off[""] = 0;
    }
    uint64_t add(const std::string& s) {
        uint64_t o = data.size();
        data.raw(s.c_str(), s.size() + 1);
        data.pad8();
        off[s] = o;
        return o;
    }
};

constexpr int GROUP_LEAF_K = 4, GROUP_INTERNAL_K = 16, ISTORE_K = 32;
constexpr size_t SNOD_SIZE = 8 + 2 * GROUP_LEAF_K * 40;
constexpr size_t GROUP_BTREE_SIZE = 24 + (2 * GROUP_INTERNAL_K + 1) * 8 + 2 * GROUP_INTERNAL_K * 8;

void sym_entry(Buf& b, uint64_t name_off, uint64_t ohdr, uint32_t cache, uint64_t btree = 0, uint64_t heap = 0) {
    b.u64(name_off);
    b.u64(ohdr);
    b.u32(cache);
    b.u32(0);
    if (cache == 1) {
        b.u64(btree);
        b.u64(heap);
    } else {
        b.zeros(16);
    }
}

struct FileWriter {
    Buf f;
    uint64_t alloc(size_t n) {
        f.pad8();
        uint64_t a = f.size();
        f.zeros(n);
        return a;
    }
    void place(uint64_t at, const Buf& b) { std::memcpy(f.b.data() + at, b.b.data(), b.size()); }
};

// group: returns (object header addr); children = (name, ohdr addr, is_group, btree, heap)
struct Child {
    std::string name;
    uint64_t ohdr;
    bool group;
    uint64_t btree, heap;
};

struct GroupAddrs {
    uint64_t btree, heap;
};

GroupAddrs write_group_index(FileWriter& w, std::vector<Child> kids) {
    std::sort(kids.begin(), kids.end(), [](const Child& a, const Child& b) { return a.name < b.name; });
    if (kids.size() > (size_t)2 * GROUP_LEAF_K) throw H5Error("too many group members");
    Heap heap;
    for (auto& k : kids) heap.add(k.name);
    Buf hdr;
    const uint64_t heap_addr = w.alloc(32);
    const uint64_t heap_data = w.alloc(heap.data.size());
    hdr.raw("HEAP", 4);
    hdr.u8(0);
    hdr.zeros(3);
    hdr.u64(heap.data.size());
    hdr.u64(UNDEF);
    hdr.u64(heap_data);
    w.place(heap_addr, hdr);
    w.place(heap_data, heap.data);
    const uint64_t snod_addr = w.alloc(SNOD_SIZE);
    Buf sn;
    sn.raw("SNOD", 4);
    sn.u8(1);
    sn.u8(0);
    sn.u16((uint16_t)kids.size());
    for (auto& k : kids) sym_entry(sn, heap.off[k.name], k.ohdr, k.group ? 1 : 0, k.btree, k.heap);
    w.place(snod_addr, sn);
    const uint64_t bt_addr = w.alloc(GROUP_BTREE_SIZE);
    Buf bt;
    bt.raw("TREE", 4);
    bt.u8(0);
    bt.u8(0);
    bt.u16(1);
    bt.u64(UNDEF);
    bt.u64(UNDEF);
    bt.u64(0);
    bt.u64(snod_addr);
    bt.u64(kids.empty() ? 0 : heap.off[kids.back().name]);
    w.place(bt_addr, bt);
    return {bt_addr, heap_addr};
}

Buf symtab_msg(const GroupAddrs& g) {
    Buf m;
    m.u64(g.btree);
    m.u64(g.heap);
    return m;
}

// chunk B-tree: leaves of up to 2K chunks, internal levels above. Keys hold
// the chunk's size (leaves), filter mask 0 and its element offsets per
// dimension plus a trailing 0 for the element-size dimension; the key after
// the last child is the last chunk's offsets advanced by one chunk in every
// dimension (rank 1: the element offset one past the last chunk).
uint64_t write_chunk_btree(FileWriter& w, const std::vector<uint64_t>& addr, const std::vector<uint32_t>& csize,
                           const std::vector<std::vector<uint64_t>>& offs, const std::vector<uint64_t>& cdims) {
    const size_t rank = cdims.size();
    const size_t key_size = 4 + 4 + 8 * (rank + 1);
    const size_t node_size = 24 + (2 * ISTORE_K + 1) * key_size + 2 * ISTORE_K * 8;
    struct Node {
        uint64_t addr;
        std::vector<uint64_t> first, last_end;  // offsets spanned
    };
    auto advance = [&](const std::vector<uint64_t>& o) {
        std::vector<uint64_t> r = o;
        for (size_t d = 0; d < rank; ++d) r[d] += cdims[d];
        return r;
    };
    std::vector<uint64_t> children = addr;
    std::vector<std::vector<uint64_t>> starts = offs, ends(addr.size());
    for (size_t i = 0; i < addr.size(); ++i) ends[i] = advance(offs[i]);
    int lvl = 0;
    std::vector<uint32_t> sizes = csize;
    while (true) {
        std::vector<Node> next;
        for (size_t b = 0; b < children.size(); b += 2 * ISTORE_K) {
            const size_t e = std::min(children.size(), b + 2 * ISTORE_K);
            const uint64_t na = w.alloc(node_size);
            Buf n;
            n.raw("TREE", 4);
            n.u8(1);
            n.u8((uint8_t)lvl);
            n.u16((uint16_t)(e - b));
            n.u64(UNDEF);
            n.u64(UNDEF);
            for (size_t i = b; i < e; ++i) {
                n.u32(lvl == 0 ? sizes[i] : 0);
                n.u32(0);
                for (size_t d = 0; d < rank; ++d) n.u64(starts[i][d]);
                n.u64(0);
                n.u64(children[i]);
            }
            n.u32(0);
            n.u32(0);
            for (size_t d = 0; d < rank; ++d) n.u64(ends[e - 1][d]);
            n.u64(0);
            w.place(na, n);
            next.push_back({na, starts[b], ends[e - 1]});
        }
        if (next.size() == 1) return next[0].addr;
        children.clear();
        starts.clear();
        ends.clear();
        for (auto& nd : next) {
            children.push_back(nd.addr);
            starts.push_back(nd.first);
            ends.push_back(nd.last_end);
        }
        ++lvl;
    }
}

// Dataset of float elements (es = 4 or 8) with dimensions `dims` (rank 1 to
// 3, row-major data). "none" is contiguous; otherwise chunked with chunk
// dimensions `cdims` (edge chunks are stored whole, zero-padded, as libhdf5
// does) and the compression's filter pipeline.
uint64_t write_dataset(FileWriter& w, const uint8_t* data, const std::vector<uint64_t>& dims,
                       const std::vector<uint64_t>& cdims, int es, const Compression& cmp) {
    Buf dspace, dtype, layout, fill, filters;
    const bool chunked = cmp.kind != Comp::None;
    const size_t rank = dims.size();
    if (rank < 1 || rank > 3 || (chunked && cdims.size() != rank)) throw H5Error("unsupported dataset rank");
    size_t n_elems = 1;
    for (auto d : dims) n_elems *= d;
    dspace.u8(1);
    dspace.u8((uint8_t)rank);
    dspace.u8(chunked ? 1 : 0);
    dspace.u8(0);
    dspace.u32(0);
    for (auto d : dims) dspace.u64(d);
    if (chunked)
        for (auto d : dims) dspace.u64(d);
    dtype_float(dtype, es);
    fill.u8(2);
    fill.u8(chunked ? 3 : 2);  // incremental / late allocation
    fill.u8(2);                // write fill value: if set by user
    fill.u8(0);                // undefined
    const size_t bytes = n_elems * (size_t)es;
    uint64_t data_addr = 0;
    if (!chunked) {
        data_addr = w.alloc(bytes);
        std::memcpy(w.f.b.data() + data_addr, data, bytes);
        layout.u8(3);
        layout.u8(1);
        layout.u64(data_addr);
        layout.u64(bytes);
    } else {
        // chunk grid, row-major (the B-tree's key order)
        std::vector<uint64_t> ng(rank);
        size_t nchunks = 1, chunk = 1;
        for (size_t d = 0; d < rank; ++d) {
            if (cdims[d] == 0 || cdims[d] > dims[d]) throw H5Error("chunk larger than the dataset");
            ng[d] = (dims[d] + cdims[d] - 1) / cdims[d];
            nchunks *= ng[d];
            chunk *= cdims[d];
        }
        std::vector<std::vector<uint64_t>> offs(nchunks, std::vector<uint64_t>(rank));
        for (size_t c = 0; c < nchunks; ++c) {
            size_t r = c;
            for (size_t d = rank; d-- > 0;) {
                offs[c][d] = (r % ng[d]) * cdims[d];
                r /= ng[d];
            }
        }
        // gather one chunk (zero padding outside the dataset)
        auto gather = [&](size_t c, uint8_t* raw) {
            const auto& o = offs[c];
            const uint64_t d1 = rank > 1 ? dims[rank - 2] : 1, d2 = dims[rank - 1];
            const uint64_t k0 = rank > 2 ? cdims[0] : 1, k1 = rank > 1 ? cdims[rank - 2] : 1, k2 = cdims[rank - 1];
            const uint64_t o0 = rank > 2 ? o[0] : 0, o1 = rank > 1 ? o[rank - 2] : 0, o2 = o[rank - 1];
            const uint64_t d0 = rank > 2 ? dims[0] : 1;
            const uint64_t run = std::min<uint64_t>(k2, d2 - o2);
            for (uint64_t a = 0; a < k0 && o0 + a < d0; ++a)
                for (uint64_t b = 0; b < k1 && o1 + b < d1; ++b)
                    std::memcpy(raw + ((a * k1 + b) * k2) * es, data + (((o0 + a) * d1 + o1 + b) * d2 + o2) * es,
                                run * es);
        };
        std::vector<uint64_t> addrs;
        std::vector<uint32_t> sizes;
        // chunks are independent: encode them on up to kEncodeThreads threads
        std::vector<std::vector<uint8_t>> enc(nchunks);
        std::vector<std::string> errs(nchunks);
        auto encode = [&](size_t c) {
            try {
                std::vector<uint8_t> raw(chunk * es, 0), tmp(chunk * es);
                gather(c, raw.data());
                if (cmp.kind == Comp::Gzip) {
                    shuffle(raw.data(), tmp.data(), raw.size(), (size_t)es);
                    enc[c] = deflate_bytes(tmp, cmp.level);
                } else {
                    enc[c] = blosc_encode(raw, es, cmp.kind == Comp::BloscZstd, cmp.level);
                }
            } catch (const std::exception& e) {
                errs[c] = e.what();
            }
        };
        const size_t nthr = std::min<size_t>(nchunks, kEncodeThreads);
        std::atomic<size_t> next{0};
        std::vector<std::thread> pool;
        for (size_t t = 1; t < nthr; ++t)
            pool.emplace_back([&]() {
                for (size_t c; (c = next++) < nchunks;) encode(c);
            });
        for (size_t c; (c = next++) < nchunks;) encode(c);
        for (auto& th : pool) th.join();
        for (auto& e : errs)
            if (!e.empty()) throw H5Error(e);
        for (size_t c = 0; c < nchunks; ++c) {
            const uint64_t a = w.alloc(enc[c].size());
            std::memcpy(w.f.b.data() + a, enc[c].data(), enc[c].size());
            addrs.push_back(a);
            sizes.push_back((uint32_t)enc[c].size());
            std::vector<uint8_t>().swap(enc[c]);
        }
        const uint64_t bt = write_chunk_btree(w, addrs, sizes, offs, cdims);
        layout.u8(3);
        layout.u8(2);
        layout.u8((uint8_t)(rank + 1));
        layout.u64(bt);
        for (auto k : cdims) layout.u32((uint32_t)k);
        layout.u32((uint32_t)es);
        filters.u8(1);
        if (cmp.kind == Comp::Gzip) {
            filters.u8(2);
            filters.zeros(6);
            filters.u16(2);  // shuffle
            filters.u16(0);
            filters.u16(1);
            filters.u16(1);
            filters.u32((uint32_t)es);
            filters.zeros(4);
            filters.u16(1);  // deflate
            filters.u16(0);
            filters.u16(1);
            filters.u16(1);
            filters.u32((uint32_t)cmp.level);
            filters.zeros(4);
        } else {
            filters.u8(1);
            filters.zeros(6);
            filters.u16(32001);  // blosc
            filters.u16(0);
            filters.u16(0);
            filters.u16(7);
            filters.u32(2);      // filter revision
            filters.u32(2);      // blosc format version
            filters.u32((uint32_t)es);
            filters.u32((uint32_t)(chunk * es));
            filters.u32((uint32_t)cmp.level);
            filters.u32(1);      // byte shuffle
            filters.u32(cmp.kind == Comp::BloscZstd ? 5 : 1);
            filters.zeros(4);
        }
    }
    std::vector<std::pair<uint16_t, Buf>> msgs = {{0x0001, dspace}, {0x0003, dtype}, {0x0005, fill}, {0x0008, layout}};
    if (chunked) msgs.push_back({0x000B, filters});
    Buf oh = object_header(msgs);
    const uint64_t a = w.alloc(oh.size());
    w.place(a, oh);
    return a;
}

// ---------------------------------------------------------------- reader
struct Reader {
    std::vector<uint8_t> f;
    const uint8_t* at(uint64_t a, size_t n) const {
        if (a == UNDEF || a + n > f.size()) throw H5Error("truncated or corrupt file (address out of range)");
        return f.data() + a;
    }
    struct Msg {
        uint16_t type;
        std::vector<uint8_t> data;
    };
    std::vector<Msg> messages(uint64_t addr) const {
        const uint8_t* h = at(addr, 16);
        if (h[0] != 1) throw H5Error("unsupported object header version");
        const int n = (int)rd(h + 2, 2);
        std::vector<Msg> out;
        std::vector<std::pair<uint64_t, uint64_t>> blocks = {{addr + 16, rd(h + 8, 4)}};
        for (size_t bi = 0; bi < blocks.size() && (int)out.size() < n; ++bi) {
            uint64_t p = blocks[bi].first, end = blocks[bi].first + blocks[bi].second;
            while (p + 8 <= end && (int)out.size() < n) {
                const uint8_t* m = at(p, 8);
                const uint16_t type = (uint16_t)rd(m, 2), sz = (uint16_t)rd(m + 2, 2);
                const uint8_t* d = at(p + 8, sz);
                if (type == 0x0010) {  // continuation
                    blocks.push_back({rd(d, 8), rd(d + 8, 8)});
                }
                out.push_back({type, std::vector<uint8_t>(d, d + sz)});
                p += 8 + sz;
            }
        }
        return out;
    }
    // members of an old-style group
    std::map<std::string, uint64_t> members(uint64_t btree, uint64_t heap) const {
        const uint8_t* hh = at(heap, 32);
        if (std::memcmp(hh, "HEAP", 4) != 0) throw H5Error("corrupt local heap");
        const uint64_t dseg = rd(hh + 24, 8), dsize = rd(hh + 8, 8);
        const uint8_t* names = at(dseg, dsize);
        std::map<std::string, uint64_t> out;
        walk_group_btree(btree, names, dsize, out);
        return out;
    }
    void walk_group_btree(uint64_t node, const uint8_t* names, uint64_t dsize,
                          std::map<std::string, uint64_t>& out) const {
        const uint8_t* t = at(node, 24);
        if (std::memcmp(t, "TREE", 4) != 0 || t[4] != 0) throw H5Error("corrupt group B-tree");
        const int level = t[5], used = (int)rd(t + 6, 2);
        const uint8_t* e = at(node + 24, (size_t)used * 16 + 8);
        for (int i = 0; i < used; ++i) {
            const uint64_t child = rd(e + 8 + 16 * i, 8);
            if (level > 0) {
                walk_group_btree(child, names, dsize, out);
                continue;
            }
            const uint8_t* s = at(child, 8);
            if (std::memcmp(s, "SNOD", 4) != 0) throw H5Error("corrupt symbol table node");
            const int ns = (int)rd(s + 6, 2);
            const uint8_t* ent = at(child + 8, (size_t)ns * 40);
            for (int k = 0; k < ns; ++k) {
                const uint64_t noff = rd(ent + 40 * k, 8);
                if (noff >= dsize) throw H5Error("corrupt link name");
                out[std::string((const char*)names + noff)] = rd(ent + 40 * k + 8, 8);
            }
        }
    }
    void collect_chunks(uint64_t node, int rank1, std::vector<std::pair<uint64_t, std::pair<uint64_t, uint32_t>>>& out,
                        std::vector<uint32_t>& masks) const {
        const size_t ks = 8 + 8 * (size_t)rank1;
        const uint8_t* t = at(node, 24);
        if (std::memcmp(t, "TREE", 4) != 0 || t[4] != 1) throw H5Error("corrupt chunk B-tree");
        const int level = t[5], used = (int)rd(t + 6, 2);
        const uint8_t* e = at(node + 24, (size_t)used * (ks + 8) + ks);
        for (int i = 0; i < used; ++i) {
            const uint8_t* key = e + i * (ks + 8);
            const uint64_t child = rd(key + ks, 8);
            if (level > 0) {
                collect_chunks(child, rank1, out, masks);
            } else {
                out.push_back({rd(key + 8, 8), {child, (uint32_t)rd(key, 4)}});
                masks.push_back((uint32_t)rd(key + 4, 4));
            }
        }
    }
};

struct Attr {
    int cls = -1;
    size_t size = 0;
    std::vector<uint8_t> value;
};

std::map<std::string, Attr> read_attrs(const std::vector<Reader::Msg>& msgs) {
    std::map<std::string, Attr> out;
    for (auto& m : msgs) {
        if (m.type != 0x000C) continue;
        const uint8_t* d = m.data.data();
        const size_t n = m.data.size();
        if (n < 8) throw H5Error("corrupt attribute");
        const int ver = d[0];
        const size_t nl = rd(d + 2, 2), dl = rd(d + 4, 2), sl = rd(d + 6, 2);
        size_t p = (ver == 1) ? 8 : (ver == 3 ? 9 : 8);
        auto adv = [&](size_t len) { return ver == 1 ? (len + 7) / 8 * 8 : len; };
        if (p + adv(nl) + adv(dl) + adv(sl) > n) throw H5Error("corrupt attribute");
        std::string name((const char*)d + p, strnlen((const char*)d + p, nl));
        p += adv(nl);
        Attr a;
        a.cls = d[p] & 0x0f;
        a.size = rd(d + p + 4, 4);
        p += adv(dl) + adv(sl);
        if (p + a.size > n) throw H5Error("corrupt attribute value");
        a.value.assign(d + p, d + p + a.size);
        out[name] = a;
    }
    return out;
}

thread_local std::string g_err;

int fail(const std::string& s, int code = -5) {
    g_err = s;
    return code;
}

// Root object header with `rmsgs`, superblock v0, then the file written
// atomically (path.tmp renamed over path). Returns 0 or fail().
int finish_file(FileWriter& w, const GroupAddrs& rg, const std::vector<std::pair<uint16_t, Buf>>& rmsgs,
                const char* path) {
    Buf roh = object_header(rmsgs);
    const uint64_t root_ohdr = w.alloc(roh.size());
    w.place(root_ohdr, roh);
    w.f.pad8();
    Buf sb;
    const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    sb.raw(sig, 8);
    sb.u8(0);
    sb.u8(0);
    sb.u8(0);
    sb.u8(0);
    sb.u8(0);
    sb.u8(8);
    sb.u8(8);
    sb.u8(0);
    sb.u16(GROUP_LEAF_K);
    sb.u16(GROUP_INTERNAL_K);
    sb.u32(0);
    sb.u64(0);
    sb.u64(UNDEF);
    sb.u64(w.f.size());
    sb.u64(UNDEF);
    sym_entry(sb, 0, root_ohdr, 1, rg.btree, rg.heap);
    w.place(0, sb);
    std::string tmp = std::string(path) + ".tmp";
    FILE* fp = std::fopen(tmp.c_str(), "wb");
    if (!fp) return fail(std::string("cannot open ") + tmp + " for writing");
    const size_t wr = std::fwrite(w.f.b.data(), 1, w.f.size(), fp);
    const int cl = std::fclose(fp);
    if (wr != w.f.size() || cl != 0) {
        std::remove(tmp.c_str());
        return fail(std::string("short write to ") + tmp);
    }
    if (std::rename(tmp.c_str(), path) != 0) return fail(std::string("cannot rename to ") + path);
    return 0;
}

}  // namespace

extern "C" {

const char* od_state_error(void) { return g_err.c_str(); }

int od_state_save(const char* path, const void* planes, int u_f64, int nx, int ny, int nz, unsigned long long step,
                  double t, double lx, double ly, double lz, const char* compression) {
    try {
        if (!path || !planes || nx <= 0 || ny <= 0 || nz <= 0) return fail("invalid arguments", -1);
        const Compression cmp = parse_compression(compression);
        const size_t npts = (size_t)nx * ny * nz * 64;
        const int es = u_f64 ? 8 : 4;
        FileWriter w;
        w.f.zeros(96);  // superblock, patched at the end
        uint64_t ds_addr[5];
        for (int v = 0; v < 5; ++v)
            ds_addr[v] = write_dataset(w, (const uint8_t*)planes + (size_t)v * npts * es, {(uint64_t)npts},
                                       {(uint64_t)std::min(npts, CHUNK_ELEMS)}, es, cmp);
        std::vector<Child> dkids;
        for (int v = 0; v < 5; ++v) dkids.push_back({VAR_NAMES[v], ds_addr[v], false, 0, 0});
        GroupAddrs dg = write_group_index(w, dkids);
        Buf doh = object_header({{0x0011, symtab_msg(dg)}});
        const uint64_t data_ohdr = w.alloc(doh.size());
        w.place(data_ohdr, doh);
        GroupAddrs rg = write_group_index(w, {{"data", data_ohdr, true, dg.btree, dg.heap}});
        // root attributes (io.rs:123-134)
        std::vector<std::pair<uint16_t, Buf>> rmsgs = {{0x0011, symtab_msg(rg)}};
        const uint64_t u64v[5] = {(uint64_t)nx, (uint64_t)ny, (uint64_t)nz, 3ull, (uint64_t)step};
        const char* u64n[5] = {"nx", "ny", "nz", "fr_order", "step"};
        for (int i = 0; i < 5; ++i) rmsgs.push_back({0x000C, attribute(u64n[i], dtype_u64, &u64v[i], 8)});
        const double f64v[4] = {t, lx, ly, lz};
        const char* f64n[4] = {"t", "lx", "ly", "lz"};
        for (int i = 0; i < 4; ++i)
            rmsgs.push_back({0x000C, attribute(f64n[i], [](Buf& b) { dtype_float(b, 8); }, &f64v[i], 8)});
        rmsgs.push_back({0x000C, attribute("u_real", dtype_str3, u_f64 ? "f64" : "f32", 3)});
        return finish_file(w, rg, rmsgs, path);
    } catch (const std::exception& e) {
        return fail(e.what());
    }
}

// Point-field file: group /data with nfields 3-D f32 datasets (row-major
// n0 x n1 x n2), no root attributes (the layout of the reference's ParaView
// companion file, scripts/h5_to_xdmf.py:130-141).
int od_fields_save(const char* path, const float* fields, int nfields, const char* const* names, long long n0,
                   long long n1, long long n2, int chunk, const char* compression) {
    try {
        if (!path || !fields || !names || nfields <= 0 || n0 <= 0 || n1 <= 0 || n2 <= 0 || chunk <= 0)
            return fail("invalid arguments", -1);
        const Compression cmp = parse_compression(compression);
        const std::vector<uint64_t> dims = {(uint64_t)n0, (uint64_t)n1, (uint64_t)n2};
        std::vector<uint64_t> cdims(3);
        for (int d = 0; d < 3; ++d) cdims[d] = std::min<uint64_t>((uint64_t)chunk, dims[d]);
        const size_t n = (size_t)n0 * n1 * n2;
        FileWriter w;
        w.f.zeros(96);  // superblock, patched at the end
        std::vector<Child> dkids;
        for (int v = 0; v < nfields; ++v) {
            if (!names[v] || !*names[v]) return fail("empty field name", -1);
            const uint64_t a = write_dataset(w, (const uint8_t*)(fields + (size_t)v * n), dims, cdims, 4, cmp);
            dkids.push_back({names[v], a, false, 0, 0});
        }
        GroupAddrs dg = write_group_index(w, dkids);
        Buf doh = object_header({{0x0011, symtab_msg(dg)}});
        const uint64_t data_ohdr = w.alloc(doh.size());
        w.place(data_ohdr, doh);
        GroupAddrs rg = write_group_index(w, {{"data", data_ohdr, true, dg.btree, dg.heap}});
        return finish_file(w, rg, {{0x0011, symtab_msg(rg)}}, path);
    } catch (const std::exception& e) {
        return fail(e.what());
    }
}

// Header of a state file: mesh, fr_order, label, time, box, precision tag.
int od_state_info(const char* path, int* nx, int* ny, int* nz, int* fr_order, unsigned long long* step, double* t,
                  double* lx, double* ly, double* lz, char* u_real4) {
    try {
        FILE* fp = path ? std::fopen(path, "rb") : nullptr;
        if (!fp) return fail(std::string("initial_state file not found: ") + (path ? path : "(null)"), -5);
        Reader r;
        std::fseek(fp, 0, SEEK_END);
        long sz = std::ftell(fp);
        std::fseek(fp, 0, SEEK_SET);
        r.f.resize(sz > 0 ? (size_t)sz : 0);
        size_t got = r.f.empty() ? 0 : std::fread(r.f.data(), 1, r.f.size(), fp);
        std::fclose(fp);
        if (got != r.f.size() || r.f.size() < 96) return fail("not an HDF5 state file (too short)");
        const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
        if (std::memcmp(r.f.data(), sig, 8) != 0) return fail("not an HDF5 file");
        const int sbv = r.f[8];
        if (sbv > 1) return fail("unsupported HDF5 superblock version " + std::to_string(sbv));
        if (r.f[13] != 8 || r.f[14] != 8) return fail("unsupported HDF5 offset / length size");
        const size_t entry = sbv == 0 ? 56 : 60;
        const uint64_t root = rd(r.f.data() + entry + 8, 8);
        auto attrs = read_attrs(r.messages(root));
        auto getu = [&](const char* k) -> uint64_t {
            auto it = attrs.find(k);
            if (it == attrs.end() || it->second.cls != 0) throw H5Error(std::string("missing attribute ") + k);
            return rd(it->second.value.data(), (int)std::min<size_t>(8, it->second.size));
        };
        auto getf = [&](const char* k) -> double {
            auto it = attrs.find(k);
            if (it == attrs.end() || it->second.cls != 1) throw H5Error(std::string("missing attribute ") + k);
            if (it->second.size == 8) {
                double d;
                std::memcpy(&d, it->second.value.data(), 8);
                return d;
            }
            float f;
            std::memcpy(&f, it->second.value.data(), 4);
            return f;
        };
        if (nx) *nx = (int)getu("nx");
        if (ny) *ny = (int)getu("ny");
        if (nz) *nz = (int)getu("nz");
        if (fr_order) *fr_order = (int)getu("fr_order");
        if (step) *step = getu("step");
        if (t) *t = getf("t");
        if (lx) *lx = getf("lx");
        if (ly) *ly = getf("ly");
        if (lz) *lz = getf("lz");
        if (u_real4) {
            auto it = attrs.find("u_real");
            if (it == attrs.end() || it->second.cls != 3) throw H5Error("missing attribute u_real");
            std::memset(u_real4, 0, 4);
            std::memcpy(u_real4, it->second.value.data(), std::min<size_t>(3, it->second.size));
        }
        return 0;
    } catch (const std::exception& e) {
        return fail(e.what());
    }
}

// Validating load (io.rs:163-234): mesh, fr_order and u_real must match; the
// five planes are read in their stored type (f64 planes stay f64).
int od_state_load(const char* path, void* planes_out, size_t bytes, int expect_u_f64, int nx, int ny, int nz,
                  unsigned long long* step, double* t) {
    try {
        int fnx, fny, fnz, fr;
        char kind[4];
        int rc = od_state_info(path, &fnx, &fny, &fnz, &fr, step, t, nullptr, nullptr, nullptr, kind);
        if (rc) return rc;
        if (fnx != nx || fny != ny || fnz != nz)
            return fail("initial_state mesh " + std::to_string(fnx) + "x" + std::to_string(fny) + "x" +
                            std::to_string(fnz) + " does not match config " + std::to_string(nx) + "x" +
                            std::to_string(ny) + "x" + std::to_string(nz) + "; refusing to load",
                        -3);
        if (fr != 3) return fail("initial_state fr_order " + std::to_string(fr) + " != configured FR_ORDER 3", -3);
        const std::string want = expect_u_f64 ? "f64" : "f32";
        if (want != kind)
            return fail(std::string("initial_state u_real '") + kind + "' does not match the configured pipeline ('" +
                            want + "'); refusing to load",
                        -3);
        const size_t npts = (size_t)nx * ny * nz * 64;
        const int es = expect_u_f64 ? 8 : 4;
        if (bytes != npts * 5 * (size_t)es) return fail("output buffer size does not match the mesh", -3);
        Reader r;
        FILE* fp = std::fopen(path, "rb");
        if (!fp) return fail(std::string("cannot open ") + path);
        std::fseek(fp, 0, SEEK_END);
        long sz = std::ftell(fp);
        std::fseek(fp, 0, SEEK_SET);
        r.f.resize((size_t)sz);
        size_t got = std::fread(r.f.data(), 1, r.f.size(), fp);
        std::fclose(fp);
        if (got != r.f.size()) return fail("short read");
        const int sbv = r.f[8];
        const size_t entry = sbv == 0 ? 56 : 60;
        const uint64_t root = rd(r.f.data() + entry + 8, 8);
        uint64_t rbt = 0, rheap = 0;
        for (auto& m : r.messages(root))
            if (m.type == 0x0011) {
                rbt = rd(m.data.data(), 8);
                rheap = rd(m.data.data() + 8, 8);
            }
        if (!rbt) return fail("root group has no symbol table (unsupported group format)");
        auto top = r.members(rbt, rheap);
        if (!top.count("data")) return fail("initial_state missing group /data");
        uint64_t dbt = 0, dheap = 0;
        for (auto& m : r.messages(top["data"]))
            if (m.type == 0x0011) {
                dbt = rd(m.data.data(), 8);
                dheap = rd(m.data.data() + 8, 8);
            }
        if (!dbt) return fail("/data has no symbol table (unsupported group format)");
        auto vars = r.members(dbt, dheap);
        for (int v = 0; v < 5; ++v) {
            if (!vars.count(VAR_NAMES[v])) return fail(std::string("initial_state missing dataset /data/") + VAR_NAMES[v]);
            uint64_t n = 0, tsize = 0;
            int tcls = -1, layout_cls = -1;
            uint64_t caddr = 0, csize = 0, cbt = 0, chunk_elems = 0;
            std::vector<std::pair<int, std::vector<uint32_t>>> filters;
            for (auto& m : r.messages(vars[VAR_NAMES[v]])) {
                const uint8_t* d = m.data.data();
                if (m.type == 0x0001) {
                    const int rank = d[1];
                    const size_t hdr = d[0] == 1 ? 8 : 4;
                    n = 1;
                    for (int k = 0; k < rank; ++k) n *= rd(d + hdr + 8 * k, 8);
                } else if (m.type == 0x0003) {
                    tcls = d[0] & 0x0f;
                    tsize = rd(d + 4, 4);
                    if (tcls == 1 && (d[1] & 1)) return fail("big-endian datasets are not supported");
                } else if (m.type == 0x0008) {
                    if (d[0] != 3) return fail("unsupported data layout message version");
                    layout_cls = d[1];
                    if (layout_cls == 1) {
                        caddr = rd(d + 2, 8);
                        csize = rd(d + 10, 8);
                    } else if (layout_cls == 2) {
                        const int dims = d[2];
                        cbt = rd(d + 3, 8);
                        chunk_elems = 1;
                        for (int k = 0; k < dims - 1; ++k) chunk_elems *= rd(d + 11 + 4 * k, 4);
                    } else {
                        return fail("unsupported data layout class");
                    }
                } else if (m.type == 0x000B) {
                    const int ver = d[0], nf = d[1];
                    size_t p = ver == 1 ? 8 : 2;
                    for (int k = 0; k < nf; ++k) {
                        const int id = (int)rd(d + p, 2);
                        size_t nl = 0;
                        p += 2;
                        if (ver == 1 || id >= 256) {
                            nl = rd(d + p, 2);
                            p += 2;
                        }
                        p += 2;  // flags
                        const int ncv = (int)rd(d + p, 2);
                        p += 2;
                        p += ver == 1 ? (nl + 7) / 8 * 8 : nl;
                        std::vector<uint32_t> cv;
                        for (int q = 0; q < ncv; ++q) cv.push_back((uint32_t)rd(d + p + 4 * q, 4));
                        p += 4 * (size_t)ncv;
                        if (ver == 1 && (ncv & 1)) p += 4;
                        filters.push_back({id, cv});
                    }
                }
            }
            if (n != npts)
                return fail(std::string("initial_state /data/") + VAR_NAMES[v] + " has " + std::to_string(n) +
                                " values, expected " + std::to_string(npts),
                            -3);
            if (tcls != 1 || (tsize != 4 && tsize != 8)) return fail("dataset is not f32 / f64");
            std::vector<uint8_t> plane(n * tsize);
            if (layout_cls == 1) {
                if (csize < plane.size()) return fail("contiguous dataset too small");
                std::memcpy(plane.data(), r.at(caddr, plane.size()), plane.size());
            } else if (layout_cls == 2) {
                std::vector<std::pair<uint64_t, std::pair<uint64_t, uint32_t>>> chunks;
                std::vector<uint32_t> masks;
                r.collect_chunks(cbt, 2, chunks, masks);
                for (size_t ci = 0; ci < chunks.size(); ++ci) {
                    const uint64_t off = chunks[ci].first;
                    const uint64_t addr = chunks[ci].second.first;
                    const uint32_t cs = chunks[ci].second.second;
                    std::vector<uint8_t> buf(r.at(addr, cs), r.at(addr, cs) + cs);
                    for (int k = (int)filters.size() - 1; k >= 0; --k) {
                        if (masks[ci] & (1u << k)) continue;
                        const int id = filters[k].first;
                        if (id == 1) {
                            buf = inflate_bytes(buf.data(), buf.size(), chunk_elems * tsize);
                        } else if (id == 2) {
                            std::vector<uint8_t> o(buf.size());
                            unshuffle(buf.data(), o.data(), buf.size(), tsize);
                            buf.swap(o);
                        } else if (id == 32001) {
                            buf = blosc_decode(buf.data(), buf.size());
                        } else {
                            return fail("unsupported HDF5 filter id " + std::to_string(id));
                        }
                    }
                    if (off >= n) continue;
                    const size_t cnt = std::min<uint64_t>(chunk_elems, n - off);
                    if (buf.size() < cnt * tsize) return fail("corrupt chunk (short)");
                    std::memcpy(plane.data() + off * tsize, buf.data(), cnt * tsize);
                }
            } else {
                return fail("dataset without a data layout");
            }
            uint8_t* dst = (uint8_t*)planes_out + (size_t)v * npts * es;
            if ((int)tsize == es) {
                std::memcpy(dst, plane.data(), plane.size());
            } else if (es == 8) {
                for (size_t i = 0; i < n; ++i) {
                    float f;
                    std::memcpy(&f, plane.data() + 4 * i, 4);
                    const double d = f;
                    std::memcpy(dst + 8 * i, &d, 8);
                }
            } else {
                for (size_t i = 0; i < n; ++i) {
                    double d;
                    std::memcpy(&d, plane.data() + 8 * i, 8);
                    const float f = (float)d;
                    std::memcpy(dst + 4 * i, &f, 4);
                }
            }
        }
        return 0;
    } catch (const std::exception& e) {
        return fail(e.what());
    }
}

}  // extern "C"
