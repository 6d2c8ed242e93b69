// gp5cu_h5.cpp - HDF5 field files in the reference's on-disk layout, without libhdf5.
//
// The reference saves a field with gp::save (src/io.cpp:56-152) and reads it with gp::load
// (:154-256): one dataset named "field" in the root group, element type
// H5Tarray_create(H5T_NATIVE_DOUBLE, 1, {2}) (a complex number as two doubles, :45), dataspace
// [nComp][Nz][Ny][Nx] (the Eigen ColMajor dims reversed, :77-90), default creation properties
// (contiguous storage).  The raw data is therefore the field's own memory order, x fastest.
//
// This file writes and reads that layout directly from the HDF5 file format specification:
//   writer  superblock version 0, version-1 object headers, the root group as a symbol table
//           (version-1 B-tree, symbol table node, local heap), a version-2 array datatype over
//           IEEE float64 little-endian, a version-1 dataspace, a version-2 fill value message and
//           a version-3 contiguous layout: the structures a default H5Fcreate/H5Dcreate2 writes;
//   reader  superblock versions 0-3 (with a user block before it), object header versions 1 and
//           2 (with continuation blocks), root groups held as a symbol table or as link messages,
//           float64 datasets whose element is a real double, an array of two doubles or a
//           compound of two doubles, contiguous or compact storage (chunked or filtered storage
//           and dense link storage are reported as unsupported).
// No GPU is involved: these are host-side file operations.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gp5cu.h"

namespace gp5 {
void set_last_error(const std::string &msg);
}

namespace {

constexpr uint64_t kUndef = ~0ull;
const unsigned char kSig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};

struct H5Error {
    int status;
    std::string msg;
};

[[noreturn]] void h5fail(int st, const std::string &m) { throw H5Error{st, m}; }

// ---- little-endian byte writer --------------------------------------------------------------
struct Out {
    std::vector<unsigned char> b;
    size_t pos() const { return b.size(); }
    void u8(unsigned v) { b.push_back((unsigned char)v); }
    void u16(unsigned v) { u8(v & 0xff), u8((v >> 8) & 0xff); }
    void u32(uint32_t v) {
        for (int i = 0; i < 4; i++) u8((v >> (8 * i)) & 0xff);
    }
    void u64(uint64_t v) {
        for (int i = 0; i < 8; i++) u8((unsigned)((v >> (8 * i)) & 0xff));
    }
    void bytes(const void *p, size_t n) {
        const unsigned char *c = static_cast<const unsigned char *>(p);
        b.insert(b.end(), c, c + n);
    }
    void zeros(size_t n) { b.insert(b.end(), n, 0); }
    void pad8() {
        while (b.size() % 8) b.push_back(0);
    }
    void put64(size_t at, uint64_t v) {
        for (int i = 0; i < 8; i++) b[at + i] = (unsigned char)((v >> (8 * i)) & 0xff);
    }
    void put32(size_t at, uint32_t v) {
        for (int i = 0; i < 4; i++) b[at + i] = (unsigned char)((v >> (8 * i)) & 0xff);
    }
    void put16(size_t at, unsigned v) {
        b[at] = v & 0xff;
        b[at + 1] = (v >> 8) & 0xff;
    }
};

// IEEE float64 little-endian datatype description (class 1, version 1): 8 + 12 bytes
void put_f64_type(Out &o) {
    o.u8(0x11);  // class 1 (floating point) | version 1 << 4
    o.u8(0x20);  // little-endian, no padding bits, mantissa normalisation 2 (implied msb)
    o.u8(63);    // sign bit position
    o.u8(0);
    o.u32(8);    // size
    o.u16(0);    // bit offset
    o.u16(64);   // bit precision
    o.u8(52);    // exponent location
    o.u8(11);    // exponent size
    o.u8(0);     // mantissa location
    o.u8(52);    // mantissa size
    o.u32(1023); // exponent bias
}

// version-1 object header message: type, size, flags, 3 reserved, data padded to 8 bytes
template <class F> void put_msg_v1(Out &o, unsigned type, unsigned flags, F &&body) {
    const size_t h = o.pos();
    o.u16(type);
    o.u16(0);
    o.u8(flags);
    o.zeros(3);
    const size_t d0 = o.pos();
    body();
    o.pad8();
    o.put16(h + 2, (unsigned)(o.pos() - d0));
}

void write_field_file(const char *path, const double *data, const int shape[3], int ncomp) {
    const uint64_t nsites = (uint64_t)shape[0] * shape[1] * shape[2];
    const uint64_t raw_bytes = nsites * (uint64_t)ncomp * 16;
    const int leafK = 4, internK = 16;
    Out o;
    // superblock, version 0 (96 bytes with the root group's symbol table entry)
    o.bytes(kSig, 8);
    o.u8(0);  // superblock version
    o.u8(0);  // free-space storage version
    o.u8(0);  // root group symbol table entry version
    o.u8(0);
    o.u8(0);  // shared header message format version
    o.u8(8);  // size of offsets
    o.u8(8);  // size of lengths
    o.u8(0);
    o.u16(leafK);
    o.u16(internK);
    o.u32(0);      // file consistency flags
    o.u64(0);      // base address
    o.u64(kUndef); // free-space info
    const size_t at_eof = o.pos();
    o.u64(0);      // end of file address (patched)
    o.u64(kUndef); // driver information block
    // root symbol table entry: name offset 0, object header, cache type 1 (B-tree, heap)
    o.u64(0);
    const size_t at_root_oh = o.pos();
    o.u64(0);
    o.u32(1);
    o.u32(0);
    const size_t at_root_scratch = o.pos();
    o.zeros(16);

    // root group object header, version 1: symbol table message (+ a NIL message)
    const uint64_t root_oh = o.pos();
    o.put64(at_root_oh, root_oh);
    o.u8(1);
    o.u8(0);
    o.u16(2);  // messages
    o.u32(1);  // reference count
    const size_t at_root_size = o.pos();
    o.u32(0);
    o.u32(0);  // pad the prefix to 16 bytes
    const size_t root_msgs = o.pos();
    size_t at_stab = 0;
    put_msg_v1(o, 0x0011, 1, [&] {
        at_stab = o.pos();
        o.u64(0);  // v1 B-tree address (patched)
        o.u64(0);  // local heap address (patched)
    });
    put_msg_v1(o, 0x0000, 0, [&] { o.zeros(8); });
    o.put32(at_root_size, (uint32_t)(o.pos() - root_msgs));

    // local heap of the root group: "" at offset 0, "field" at offset 8
    const uint64_t heap = o.pos();
    o.bytes("HEAP", 4);
    o.u8(0);
    o.zeros(3);
    o.u64(16);  // data segment size
    o.u64(1);   // free list: none (offset 1 marks the end)
    const size_t at_heap_data = o.pos();
    o.u64(0);
    const uint64_t heap_data = o.pos();
    o.put64(at_heap_data, heap_data);
    o.zeros(8);
    o.bytes("field\0\0\0", 8);

    // version-1 B-tree (group nodes), one leaf entry pointing at the symbol table node; the
    // node is reserved at its full size (2K children, 2K+1 keys)
    const uint64_t btree = o.pos();
    o.bytes("TREE", 4);
    o.u8(0);  // node type: group
    o.u8(0);  // level: leaf
    o.u16(1); // entries used
    o.u64(kUndef);
    o.u64(kUndef);
    o.u64(0);  // key 0: heap offset of ""
    const size_t at_snod_ptr = o.pos();
    o.u64(0);  // child 0: symbol table node (patched)
    o.u64(8);  // key 1: heap offset of "field", the largest name in the child
    o.zeros((size_t)(2 * internK - 1) * 8 + (size_t)(2 * internK + 1 - 2) * 8);
    o.put64(at_stab, btree);
    o.put64(at_stab + 8, heap);
    o.put64(at_root_scratch, btree);
    o.put64(at_root_scratch + 8, heap);

    // symbol table node with the one entry "field" (reserved for 2 * leafK entries)
    const uint64_t snod = o.pos();
    o.put64(at_snod_ptr, snod);
    o.bytes("SNOD", 4);
    o.u8(1);
    o.u8(0);
    o.u16(1);
    o.u64(8);  // name "field"
    const size_t at_ds_oh = o.pos();
    o.u64(0);  // object header (patched)
    o.u32(0);  // cache type: none
    o.u32(0);
    o.zeros(16);
    o.zeros((size_t)(2 * leafK - 1) * 40);

    // dataset object header, version 1
    const uint64_t ds = o.pos();
    o.put64(at_ds_oh, ds);
    o.u8(1);
    o.u8(0);
    o.u16(4);
    o.u32(1);
    const size_t at_ds_size = o.pos();
    o.u32(0);
    o.u32(0);
    const size_t ds_msgs = o.pos();
    // fill value (new form), version 2: allocation late, written if set, default value
    put_msg_v1(o, 0x0005, 1, [&] {
        o.u8(2);
        o.u8(2);
        o.u8(2);
        o.u8(1);
        o.u32(0);
    });
    // datatype: array (class 10), version 2, of 2 x float64, 16 bytes
    put_msg_v1(o, 0x0003, 1, [&] {
        o.u8(0x2a);
        o.zeros(3);
        o.u32(16);
        o.u8(1);  // array rank
        o.zeros(3);
        o.u32(2);  // dimension
        o.u32(0);  // permutation index
        put_f64_type(o);
    });
    // dataspace, version 1: [ncomp][nz][ny][nx]
    put_msg_v1(o, 0x0001, 0, [&] {
        o.u8(1);
        o.u8(4);
        o.u8(0);
        o.u8(0);
        o.u32(0);
        o.u64((uint64_t)ncomp);
        o.u64((uint64_t)shape[2]);
        o.u64((uint64_t)shape[1]);
        o.u64((uint64_t)shape[0]);
    });
    // layout, version 3: contiguous, raw data address and size
    size_t at_raw = 0;
    put_msg_v1(o, 0x0008, 1, [&] {
        o.u8(3);
        o.u8(1);
        at_raw = o.pos();
        o.u64(0);
        o.u64(raw_bytes);
    });
    o.put32(at_ds_size, (uint32_t)(o.pos() - ds_msgs));
    o.pad8();
    const uint64_t raw = o.pos();
    o.put64(at_raw, raw);
    o.put64(at_eof, raw + raw_bytes);

    FILE *fh = std::fopen(path, "wb");
    if (!fh) h5fail(GP5_ERR_IO, std::string("cannot create ") + path);
    bool ok = std::fwrite(o.b.data(), 1, o.b.size(), fh) == o.b.size();
    // the payload is the field's memory order (x fastest, components slowest)
    ok = ok && std::fwrite(data, 1, (size_t)raw_bytes, fh) == (size_t)raw_bytes;
    ok = (std::fclose(fh) == 0) && ok;
    if (!ok) h5fail(GP5_ERR_IO, std::string("write error on ") + path);
}

// ---- reader -----------------------------------------------------------------------------------
struct File {
    FILE *fh = nullptr;
    uint64_t size = 0;
    uint64_t base = 0;  // absolute position of address 0
    int osz = 8, lsz = 8;
    uint64_t root_oh = kUndef;
    std::string path;
    ~File() {
        if (fh) std::fclose(fh);
    }
    std::vector<unsigned char> read_abs(uint64_t pos, uint64_t n) const {
        if (pos > size || n > size - pos) h5fail(GP5_ERR_IO, path + ": truncated HDF5 structure");
        std::vector<unsigned char> v((size_t)n);
        if (n && (fseeko(fh, (off_t)pos, SEEK_SET) != 0 || std::fread(v.data(), 1, (size_t)n, fh) != n))
            h5fail(GP5_ERR_IO, path + ": read error");
        return v;
    }
    std::vector<unsigned char> read(uint64_t addr, uint64_t n) const {
        if (addr == kUndef) h5fail(GP5_ERR_IO, path + ": undefined address");
        return read_abs(base + addr, n);
    }
};

struct Rd {
    const std::vector<unsigned char> &b;
    size_t p;
    const File &f;
    void need(size_t n) const {
        if (p + n > b.size()) h5fail(GP5_ERR_IO, f.path + ": malformed HDF5 structure");
    }
    uint64_t un(int n) {
        need((size_t)n);
        uint64_t v = 0;
        for (int i = 0; i < n; i++) v |= (uint64_t)b[p + i] << (8 * i);
        p += (size_t)n;
        return v;
    }
    unsigned u8() { return (unsigned)un(1); }
    unsigned u16() { return (unsigned)un(2); }
    uint32_t u32() { return (uint32_t)un(4); }
    // an address; all ones (of the file's offset size) is the undefined address
    uint64_t off() {
        const uint64_t v = un(f.osz);
        return (f.osz < 8 && v == ((1ull << (8 * f.osz)) - 1)) ? kUndef : v;
    }
    uint64_t len() { return un(f.lsz); }
    void skip(size_t n) {
        need(n);
        p += n;
    }
};

void open_file(File &f, const char *path) {
    f.path = path;
    f.fh = std::fopen(path, "rb");
    if (!f.fh) h5fail(GP5_ERR_IO, std::string("cannot open ") + path);
    fseeko(f.fh, 0, SEEK_END);
    f.size = (uint64_t)ftello(f.fh);
    // the superblock sits at 0, 512, 1024, 2048, ... (after an optional user block)
    uint64_t at = kUndef;
    for (uint64_t q = 0; q + 8 <= f.size; q = q ? q * 2 : 512) {
        const auto s = f.read_abs(q, 8);
        if (std::memcmp(s.data(), kSig, 8) == 0) {
            at = q;
            break;
        }
    }
    if (at == kUndef) h5fail(GP5_ERR_IO, f.path + ": not an HDF5 file (no superblock signature)");
    const auto hd = f.read_abs(at, std::min<uint64_t>(f.size - at, 256));
    Rd r{hd, 8, f};
    const unsigned ver = r.u8();
    if (ver <= 1) {
        r.skip(4);  // free-space, root entry, reserved, shared header versions
        f.osz = (int)r.u8();
        f.lsz = (int)r.u8();
        r.skip(1);
        if ((f.osz != 2 && f.osz != 4 && f.osz != 8) || (f.lsz != 2 && f.lsz != 4 && f.lsz != 8))
            h5fail(GP5_ERR_UNSUPPORTED, f.path + ": unsupported offset/length sizes");
        r.skip(2 + 2 + 4);  // leaf K, internal K, flags
        if (ver == 1) r.skip(4);
        const uint64_t base = r.off();
        r.off();  // free-space info
        r.off();  // end of file
        r.off();  // driver information
        f.base = base == kUndef ? at : base;
        r.off();  // root entry: link name offset
        f.root_oh = r.off();
    } else if (ver == 2 || ver == 3) {
        f.osz = (int)r.u8();
        f.lsz = (int)r.u8();
        r.skip(1);  // flags
        const uint64_t base = r.off();
        r.off();  // superblock extension
        r.off();  // end of file
        f.base = base == kUndef ? at : base;
        f.root_oh = r.off();
    } else {
        h5fail(GP5_ERR_UNSUPPORTED, f.path + ": superblock version " + std::to_string(ver) + " is not supported");
    }
}

struct Msg {
    unsigned type;
    std::vector<unsigned char> data;
};

// All messages of an object header (versions 1 and 2), continuation blocks followed.
std::vector<Msg> read_header(const File &f, uint64_t addr) {
    std::vector<Msg> out;
    const auto first = f.read(addr, 4);
    struct Block {
        uint64_t addr, len;
    };
    std::vector<Block> todo;
    bool v2 = std::memcmp(first.data(), "OHDR", 4) == 0;
    if (!v2) {
        const auto h = f.read(addr, 16);
        Rd r{h, 0, f};
        const unsigned ver = r.u8();
        if (ver != 1) h5fail(GP5_ERR_UNSUPPORTED, f.path + ": object header version " + std::to_string(ver));
        r.skip(1);
        const unsigned nmsg = r.u16();
        r.skip(4);
        const uint32_t sz = r.u32();
        todo.push_back({addr + 16, sz});
        size_t got = 0;
        for (size_t k = 0; k < todo.size() && got < nmsg; k++) {
            const auto blk = f.read(todo[k].addr, todo[k].len);
            Rd m{blk, 0, f};
            while (m.p + 8 <= blk.size() && got < nmsg) {
                const unsigned type = m.u16(), size = m.u16();
                m.skip(4);
                m.need(size);
                Msg msg{type, std::vector<unsigned char>(blk.begin() + (long)m.p, blk.begin() + (long)(m.p + size))};
                m.skip(size);
                got++;
                if (type == 0x0010) {
                    Rd c{msg.data, 0, f};
                    const uint64_t a = c.off(), l = c.len();
                    todo.push_back({a, l});
                }
                out.push_back(std::move(msg));
            }
        }
        return out;
    }
    // version 2: "OHDR", version, flags, [times], [attribute limits], chunk-0 size, messages,
    // checksum; continuation blocks "OCHK", messages, checksum
    const auto h = f.read(addr, std::min<uint64_t>(64, f.size - f.base - addr));
    Rd r{h, 4, f};
    const unsigned ver = r.u8();
    if (ver != 2) h5fail(GP5_ERR_UNSUPPORTED, f.path + ": object header version " + std::to_string(ver));
    const unsigned flags = r.u8();
    if (flags & 0x20) r.skip(16);
    if (flags & 0x10) r.skip(4);
    const uint64_t c0 = r.un(1 << (flags & 3));
    const bool crt = (flags & 0x04) != 0;
    todo.push_back({addr + r.p, c0});
    for (size_t k = 0; k < todo.size(); k++) {
        const auto blk = f.read(todo[k].addr, todo[k].len);
        Rd m{blk, 0, f};
        if (k > 0) {
            if (blk.size() < 8 || std::memcmp(blk.data(), "OCHK", 4) != 0)
                h5fail(GP5_ERR_IO, f.path + ": bad object header continuation block");
            m.p = 4;
        }
        const size_t end = k > 0 ? blk.size() - 4 : blk.size();
        const size_t hsz = crt ? 6 : 4;
        while (m.p + hsz <= end) {
            const unsigned type = m.u8(), size = m.u16();
            m.skip(1);
            if (crt) m.skip(2);
            if (m.p + size > end) break;
            Msg msg{type, std::vector<unsigned char>(blk.begin() + (long)m.p, blk.begin() + (long)(m.p + size))};
            m.skip(size);
            if (type == 0x0010) {
                Rd c{msg.data, 0, f};
                const uint64_t a = c.off(), l = c.len();
                todo.push_back({a, l});
            }
            out.push_back(std::move(msg));
        }
    }
    return out;
}

// Walks a version-1 group B-tree and collects (name, object header) of every entry.
void walk_group_btree(const File &f, uint64_t node, const std::vector<unsigned char> &heap,
                      std::vector<std::pair<std::string, uint64_t>> &out, int depth) {
    if (depth > 32) h5fail(GP5_ERR_IO, f.path + ": group B-tree too deep");
    const auto hd = f.read(node, 8);
    if (std::memcmp(hd.data(), "TREE", 4) != 0) h5fail(GP5_ERR_IO, f.path + ": bad group B-tree node");
    const unsigned type = hd[4], level = hd[5], used = (unsigned)hd[6] | ((unsigned)hd[7] << 8);
    if (type != 0) h5fail(GP5_ERR_IO, f.path + ": group B-tree node of the wrong type");
    const uint64_t n = 8 + 2 * (uint64_t)f.osz + (uint64_t)used * (f.lsz + f.osz) + f.lsz;
    const auto b = f.read(node, n);
    Rd r{b, 8 + 2 * (size_t)f.osz, f};
    for (unsigned e = 0; e < used; e++) {
        r.len();  // key
        const uint64_t child = r.off();
        if (level > 0) {
            walk_group_btree(f, child, heap, out, depth + 1);
            continue;
        }
        const auto sh = f.read(child, 8);
        if (std::memcmp(sh.data(), "SNOD", 4) != 0) h5fail(GP5_ERR_IO, f.path + ": bad symbol table node");
        const unsigned nsym = (unsigned)sh[6] | ((unsigned)sh[7] << 8);
        const uint64_t esz = 2 * (uint64_t)f.osz + 24;
        const auto sb = f.read(child + 8, nsym * esz);
        Rd s{sb, 0, f};
        for (unsigned k = 0; k < nsym; k++) {
            const uint64_t name_off = s.off(), oh = s.off();
            s.skip(24);
            if (name_off >= heap.size()) h5fail(GP5_ERR_IO, f.path + ": symbol name outside the local heap");
            const char *c = reinterpret_cast<const char *>(heap.data() + name_off);
            out.emplace_back(std::string(c, strnlen(c, heap.size() - name_off)), oh);
        }
    }
}

// (name, object header address) of every member of the root group.
std::vector<std::pair<std::string, uint64_t>> root_members(const File &f) {
    std::vector<std::pair<std::string, uint64_t>> out;
    for (const Msg &m : read_header(f, f.root_oh)) {
        if (m.type == 0x0011) {  // symbol table: v1 B-tree + local heap
            Rd r{m.data, 0, f};
            const uint64_t btree = r.off(), heap = r.off();
            const auto hh = f.read(heap, 8 + 2 * (uint64_t)f.lsz + f.osz);
            if (std::memcmp(hh.data(), "HEAP", 4) != 0) h5fail(GP5_ERR_IO, f.path + ": bad local heap");
            Rd h{hh, 8, f};
            const uint64_t dsize = h.len();
            h.len();
            const uint64_t daddr = h.off();
            walk_group_btree(f, btree, f.read(daddr, dsize), out, 0);
        } else if (m.type == 0x0006) {  // link message (compact group storage)
            Rd r{m.data, 0, f};
            r.u8();  // version
            const unsigned flags = r.u8();
            unsigned ltype = 0;
            if (flags & 0x08) ltype = r.u8();
            if (flags & 0x04) r.skip(8);
            if (flags & 0x10) r.skip(1);
            const uint64_t nlen = r.un(1 << (flags & 3));
            r.need((size_t)nlen);
            std::string name(reinterpret_cast<const char *>(m.data.data() + r.p), (size_t)nlen);
            r.skip((size_t)nlen);
            if (ltype == 0) out.emplace_back(name, r.off());
        } else if (m.type == 0x0002) {  // link info: dense storage is in a fractal heap
            Rd r{m.data, 0, f};
            r.u8();
            const unsigned flags = r.u8();
            if (flags & 1) r.skip(8);
            if (r.off() != kUndef)
                h5fail(GP5_ERR_UNSUPPORTED, f.path + ": root group links in dense storage are not supported");
        }
    }
    return out;
}

struct DatasetInfo {
    std::vector<uint64_t> dims;
    int complex_elems = 0;  // element = 2 doubles
    uint64_t raw_addr = kUndef, raw_size = 0;
    std::vector<unsigned char> compact;
    bool is_compact = false;
};

bool is_f64_le(Rd &r) {
    const unsigned cv = r.u8();
    const unsigned bf0 = r.u8();
    r.skip(2);
    const uint32_t size = r.u32();
    if ((cv & 0x0f) != 1 || size != 8 || (bf0 & 1)) return false;
    const unsigned off = r.u16(), prec = r.u16();
    r.skip(8);
    return off == 0 && prec == 64;
}

// Element type of a dataset: 1 = real double, 2 = two doubles (array or compound); 0 otherwise.
int element_doubles(const File &f, const std::vector<unsigned char> &d) {
    Rd r{d, 0, f};
    const unsigned cv = d.size() ? d[0] : 0;
    const unsigned cls = cv & 0x0f, ver = cv >> 4;
    if (cls == 1) return is_f64_le(r) ? 1 : 0;
    if (cls == 10) {  // array
        r.skip(4);
        const uint32_t size = r.u32();
        const unsigned rank = r.u8();
        if (ver < 3) r.skip(3);
        uint64_t n = 1;
        for (unsigned k = 0; k < rank; k++) n *= r.u32();
        if (ver < 3) r.skip(4 * (size_t)rank);
        return (n == 2 && size == 16 && is_f64_le(r)) ? 2 : 0;
    }
    if (cls == 6) {  // compound of two doubles at offsets 0 and 8
        const unsigned nm = (unsigned)d[1] | ((unsigned)d[2] << 8);
        r.skip(4);
        const uint32_t size = r.u32();
        if (nm != 2 || size != 16) return 0;
        for (unsigned k = 0; k < 2; k++) {
            const char *c = reinterpret_cast<const char *>(d.data() + r.p);
            const size_t nl = strnlen(c, d.size() - r.p);
            if (ver < 3) r.skip((nl + 8) / 8 * 8);
            else r.skip(nl + 1);
            const uint64_t off = ver < 3 ? r.u32() : r.un(size < 256 ? 1 : (size < 65536 ? 2 : 4));
            if (ver == 1) r.skip(28);
            if (off != 8 * k || !is_f64_le(r)) return 0;
        }
        return 2;
    }
    return 0;
}

DatasetInfo dataset_info(const File &f, const std::string &name) {
    const auto members = root_members(f);
    uint64_t oh = kUndef;
    for (const auto &m : members)
        if (m.first == name) oh = m.second;
    if (oh == kUndef) {
        std::string list;
        for (const auto &m : members) list += (list.empty() ? "" : ", ") + m.first;
        h5fail(GP5_ERR_ARG, f.path + ": no dataset '" + name + "' in the root group (members: " + list + ")");
    }
    DatasetInfo info;
    bool have_space = false, have_type = false, have_layout = false;
    for (const Msg &m : read_header(f, oh)) {
        Rd r{m.data, 0, f};
        if (m.type == 0x0001) {
            const unsigned ver = r.u8(), rank = r.u8();
            r.u8();  // flags
            if (ver == 1) r.skip(5);
            else r.skip(1);
            info.dims.clear();
            for (unsigned k = 0; k < rank; k++) info.dims.push_back(r.len());
            have_space = true;
        } else if (m.type == 0x0003) {
            info.complex_elems = element_doubles(f, m.data);
            if (info.complex_elems == 0)
                h5fail(GP5_ERR_UNSUPPORTED, f.path + ": dataset '" + name + "' is not float64 (real or complex)");
            info.complex_elems = info.complex_elems == 2;
            have_type = true;
        } else if (m.type == 0x0008) {
            const unsigned ver = r.u8();
            if (ver == 1 || ver == 2) {
                const unsigned rank = r.u8(), cls = r.u8();
                r.skip(5);
                if (cls == 1) {
                    info.raw_addr = r.off();
                    uint64_t n = 1;
                    for (unsigned k = 0; k < rank; k++) n *= r.u32();
                    info.raw_size = n;  // dims include the element size
                } else if (cls == 0) {
                    r.skip(4 * (size_t)rank);
                    const uint32_t cs = r.u32();
                    r.need(cs);
                    info.compact.assign(m.data.begin() + (long)r.p, m.data.begin() + (long)(r.p + cs));
                    info.is_compact = true;
                } else {
                    h5fail(GP5_ERR_UNSUPPORTED, f.path + ": chunked storage is not supported");
                }
            } else if (ver == 3 || ver == 4) {
                const unsigned cls = r.u8();
                if (cls == 1) {
                    info.raw_addr = r.off();
                    info.raw_size = r.len();
                } else if (cls == 0) {
                    const unsigned cs = r.u16();
                    r.need(cs);
                    info.compact.assign(m.data.begin() + (long)r.p, m.data.begin() + (long)(r.p + cs));
                    info.is_compact = true;
                } else {
                    h5fail(GP5_ERR_UNSUPPORTED, f.path + ": chunked or virtual storage is not supported");
                }
            } else {
                h5fail(GP5_ERR_UNSUPPORTED, f.path + ": layout message version " + std::to_string(ver));
            }
            have_layout = true;
        } else if (m.type == 0x000b) {
            h5fail(GP5_ERR_UNSUPPORTED, f.path + ": filtered (compressed) datasets are not supported");
        }
    }
    if (!have_space || !have_type || !have_layout)
        h5fail(GP5_ERR_IO, f.path + ": '" + name + "' is not a dataset with a dataspace, datatype and layout");
    return info;
}

uint64_t elements(const DatasetInfo &d) {
    uint64_t n = 1;
    for (uint64_t v : d.dims) n *= v;
    return n;
}

void read_values(const File &f, const DatasetInfo &d, double *out, uint64_t count) {
    const uint64_t bytes = count * 8;
    if (d.is_compact) {
        if (d.compact.size() < bytes) h5fail(GP5_ERR_IO, f.path + ": compact data shorter than its dataspace");
        std::memcpy(out, d.compact.data(), (size_t)bytes);
        return;
    }
    if (d.raw_addr == kUndef) {  // never written: the default fill value
        std::memset(out, 0, (size_t)bytes);
        return;
    }
    if (d.raw_size < bytes) h5fail(GP5_ERR_IO, f.path + ": contiguous storage shorter than its dataspace");
    const uint64_t pos = f.base + d.raw_addr;
    if (pos > f.size || bytes > f.size - pos) h5fail(GP5_ERR_IO, f.path + ": truncated dataset");
    if (fseeko(f.fh, (off_t)pos, SEEK_SET) != 0 || std::fread(out, 1, (size_t)bytes, f.fh) != bytes)
        h5fail(GP5_ERR_IO, f.path + ": read error");
}

// [ncomp][nz][ny][nx] complex dataset "field" -> shape (x, y, z) and component count
void field_shape(const File &f, const DatasetInfo &d, int shape[3], int *ncomp) {
    if (!d.complex_elems || d.dims.size() != 4)
        h5fail(GP5_ERR_ARG, f.path + ": 'field' must be a rank-4 complex dataset [nComp][Nz][Ny][Nx]");
    for (int k = 0; k < 4; k++)
        if (d.dims[k] < 1 || d.dims[k] > (1u << 30)) h5fail(GP5_ERR_ARG, f.path + ": 'field' dimensions out of range");
    *ncomp = (int)d.dims[0];
    shape[0] = (int)d.dims[3];
    shape[1] = (int)d.dims[2];
    shape[2] = (int)d.dims[1];
}

int fail_h5(const H5Error &e) {
    gp5::set_last_error(e.msg);
    return e.status;
}

}  // namespace

extern "C" {

int gp5cu_h5_save_field(const char *path, const double *host_c128, const int shape[3], int ncomp) {
    if (!path || !host_c128 || !shape) return fail_h5({GP5_ERR_ARG, "NULL argument"});
    if (ncomp < 1 || ncomp > 2) return fail_h5({GP5_ERR_ARG, "ncomp must be 1 or 2"});
    for (int d = 0; d < 3; d++)
        if (shape[d] < 1) return fail_h5({GP5_ERR_ARG, "shape entries must be positive"});
    try {
        write_field_file(path, host_c128, shape, ncomp);
    } catch (const H5Error &e) {
        return fail_h5(e);
    }
    return GP5_OK;
}

int gp5cu_h5_field_shape(const char *path, int shape[3], int *ncomp) {
    if (!path || !shape || !ncomp) return fail_h5({GP5_ERR_ARG, "NULL argument"});
    try {
        File f;
        open_file(f, path);
        field_shape(f, dataset_info(f, "field"), shape, ncomp);
    } catch (const H5Error &e) {
        return fail_h5(e);
    }
    return GP5_OK;
}

int gp5cu_h5_load_field(const char *path, double *host_c128, const int shape[3], int ncomp) {
    if (!path || !host_c128 || !shape) return fail_h5({GP5_ERR_ARG, "NULL argument"});
    try {
        File f;
        open_file(f, path);
        const DatasetInfo d = dataset_info(f, "field");
        int s[3], nc = 0;
        field_shape(f, d, s, &nc);
        if (nc != ncomp || s[0] != shape[0] || s[1] != shape[1] || s[2] != shape[2])
            h5fail(GP5_ERR_ARG, f.path + ": 'field' is " + std::to_string(nc) + " x " + std::to_string(s[2]) + " x " +
                                    std::to_string(s[1]) + " x " + std::to_string(s[0]) +
                                    " ([nComp][Nz][Ny][Nx]), not the requested " + std::to_string(ncomp) + " x " +
                                    std::to_string(shape[2]) + " x " + std::to_string(shape[1]) + " x " +
                                    std::to_string(shape[0]));
        read_values(f, d, host_c128, 2 * elements(d));
    } catch (const H5Error &e) {
        return fail_h5(e);
    }
    return GP5_OK;
}

int gp5cu_h5_dataset_info(const char *path, const char *name, int *rank, long long dims[8], int *complex_elems) {
    if (!path || !name || !rank || !dims || !complex_elems) return fail_h5({GP5_ERR_ARG, "NULL argument"});
    try {
        File f;
        open_file(f, path);
        const DatasetInfo d = dataset_info(f, name);
        if (d.dims.size() > 8) h5fail(GP5_ERR_UNSUPPORTED, f.path + ": rank above 8");
        *rank = (int)d.dims.size();
        for (size_t k = 0; k < d.dims.size(); k++) dims[k] = (long long)d.dims[k];
        *complex_elems = d.complex_elems;
    } catch (const H5Error &e) {
        return fail_h5(e);
    }
    return GP5_OK;
}

int gp5cu_h5_read_dataset(const char *path, const char *name, double *out, long long count) {
    if (!path || !name || !out || count < 0) return fail_h5({GP5_ERR_ARG, "invalid argument"});
    try {
        File f;
        open_file(f, path);
        const DatasetInfo d = dataset_info(f, name);
        const uint64_t n = elements(d) * (d.complex_elems ? 2 : 1);
        if ((uint64_t)count != n)
            h5fail(GP5_ERR_ARG, f.path + ": '" + name + "' holds " + std::to_string(n) + " doubles, not " +
                                    std::to_string(count));
        read_values(f, d, out, n);
    } catch (const H5Error &e) {
        return fail_h5(e);
    }
    return GP5_OK;
}

}  // extern "C"
