// HDF5 output at the boundary: the datasets of the Python reference's
// saveHDF5 (CODE/Python/simLB/LBM.py:516-567) - rho, T, ux, uy as {Nx, Ny}
// arrays over [x*Ny + y], the scalars t, gamma, R, T_ref, rho_ref, dx, dy
// (dx, dy as arrays when the cells are not uniform), Nx, Ny and, with the
// distributions, f and h as {Nx, Ny, 13} over [(x*Ny + y)*13 + i].  All
// little-endian IEEE doubles except Nx and Ny (64-bit integers, as numpy
// stores Python ints).
//
// The file is written from the published HDF5 file-format specification
// with the oldest structures the HDF5 library reads: superblock version 0
// with 8-byte offsets and lengths; the root group as a version-1 object
// header holding a symbol-table message, the group's local heap of link
// names, one version-1 B-tree node (group node, level 0) and one symbol
// table node; every dataset a version-1 object header with a version-1
// dataspace, a floating-point or fixed-point datatype and a contiguous
// data layout (version 3), its raw data after the headers.
#include "lbm_hdf5.h"
#include "lbm_host.h"
#include "../../include/uq_lbm.h"

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace uqlbm {
namespace {

constexpr int NDIR = 13;             // D2Q13 velocities per node
constexpr uint64_t UNDEF = ~0ull;    // the undefined address
constexpr uint64_t HEAP_FREE_NULL = 1;  // "no free block" in a local heap
constexpr int LEAF_K = 8;            // group leaf node K: 2K = 16 links in one symbol table node
constexpr int INTERNAL_K = 16;       // group internal node K
constexpr size_t ENTRY = 40;         // symbol table entry (8-byte offsets and lengths)
constexpr size_t BTREE_NODE = 24 + 2 * INTERNAL_K * 8 + (2 * INTERNAL_K + 1) * 8;
constexpr size_t SNOD_NODE = 8 + 2 * LEAF_K * ENTRY;

size_t pad8(size_t n) { return (n + 7) / 8 * 8; }

struct Out {
    std::vector<uint8_t> b;
    size_t pos() const { return b.size(); }
    void put(uint64_t v, int n)
    {
        for (int i = 0; i < n; ++i) b.push_back((uint8_t)(v >> (8 * i)));
    }
    void zeros(size_t n) { b.insert(b.end(), n, 0); }
    void bytes(const void *p, size_t n)
    {
        const uint8_t *q = static_cast<const uint8_t *>(p);
        b.insert(b.end(), q, q + n);
    }
    void align8() { zeros(pad8(pos()) - pos()); }
    void patch(size_t at, uint64_t v, int n)
    {
        for (int i = 0; i < n; ++i) b[at + i] = (uint8_t)(v >> (8 * i));
    }
};

struct Dataset {
    std::string name;
    bool integer;                // int64 instead of double
    std::vector<uint64_t> dims;  // empty: scalar
    std::vector<uint8_t> data;   // raw little-endian bytes
};

Dataset doubles(const char *name, std::vector<uint64_t> dims, const double *p, size_t n)
{
    Dataset d{name, false, std::move(dims), {}};
    d.data.resize(n * 8);
    std::memcpy(d.data.data(), p, n * 8);
    return d;
}

Dataset scalar(const char *name, double v) { return doubles(name, {}, &v, 1); }

Dataset integer(const char *name, long long v)
{
    Dataset d{name, true, {}, {}};
    d.data.resize(8);
    std::memcpy(d.data.data(), &v, 8);
    return d;
}

// one header message of a version-1 object header (data padded to 8 bytes)
void message(Out &o, int type, const Out &data)
{
    o.put(type, 2);
    o.put(pad8(data.b.size()), 2);
    o.put(0, 1);  // flags
    o.zeros(3);
    o.bytes(data.b.data(), data.b.size());
    o.zeros(pad8(data.b.size()) - data.b.size());
}

// version-1 object header: 16-byte prefix, then the messages
void object_header(Out &o, const std::vector<std::pair<int, Out>> &msgs)
{
    size_t body = 0;
    for (const auto &m : msgs) body += 8 + pad8(m.second.b.size());
    o.put(1, 1);  // version
    o.put(0, 1);
    o.put(msgs.size(), 2);
    o.put(1, 4);  // object reference count
    o.put(body, 4);
    o.zeros(4);   // the prefix is aligned to 8 bytes
    for (const auto &m : msgs) message(o, m.first, m.second);
}

void write_file(const char *path, std::vector<Dataset> ds)
{
    if (ds.size() > 2 * LEAF_K) throw LbmError(LBM_ERR_INVALID, "too many datasets for one symbol table node");
    // links in name order (strcmp), the order of a symbol table node
    std::sort(ds.begin(), ds.end(), [](const Dataset &a, const Dataset &b) { return a.name < b.name; });
    // the group's local heap: the empty name at 0, then every name, each
    // null-terminated and padded to 8 bytes
    std::vector<uint8_t> heap(8, 0);
    std::vector<uint64_t> name_off;
    for (const Dataset &d : ds) {
        name_off.push_back(heap.size());
        heap.insert(heap.end(), d.name.begin(), d.name.end());
        heap.push_back(0);
        heap.resize(pad8(heap.size()), 0);
    }

    Out o;
    // superblock version 0
    const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    o.bytes(sig, 8);
    o.put(0, 1);  // superblock version
    o.put(0, 1);  // free-space storage version
    o.put(0, 1);  // root group symbol table entry version
    o.put(0, 1);
    o.put(0, 1);  // shared header message format version
    o.put(8, 1);  // size of offsets
    o.put(8, 1);  // size of lengths
    o.put(0, 1);
    o.put(LEAF_K, 2);
    o.put(INTERNAL_K, 2);
    o.put(0, 4);  // file consistency flags
    o.put(0, 8);  // base address
    o.put(UNDEF, 8);  // free-space info
    const size_t at_eof = o.pos();
    o.put(0, 8);      // end of file address (patched)
    o.put(UNDEF, 8);  // driver information block
    // root group symbol table entry, with the cached B-tree and heap addresses
    o.put(0, 8);  // link name offset
    const size_t at_root_oh = o.pos();
    o.put(0, 8);
    o.put(1, 4);  // cache type: symbol table
    o.put(0, 4);
    const size_t at_root_bt = o.pos();
    o.put(0, 8);
    const size_t at_root_heap = o.pos();
    o.put(0, 8);

    // root group object header: one symbol table message
    o.align8();
    const size_t root_oh = o.pos();
    Out stab;
    const size_t stab_bt = 0, stab_heap = 8;  // offsets within the message data
    stab.put(0, 8);
    stab.put(0, 8);
    object_header(o, {{0x0011, stab}});
    const size_t at_msg_data = root_oh + 16 + 8;  // first message's data

    // local heap: header, then its data segment
    o.align8();
    const size_t heap_hdr = o.pos();
    o.bytes("HEAP", 4);
    o.put(0, 1);
    o.zeros(3);
    o.put(heap.size(), 8);
    o.put(HEAP_FREE_NULL, 8);
    o.put(heap_hdr + 32, 8);
    o.bytes(heap.data(), heap.size());

    // B-tree node (group node, leaf level): key 0 the empty name, child 0
    // the symbol table node, key 1 the last name in it
    o.align8();
    const size_t btree = o.pos();
    o.bytes("TREE", 4);
    o.put(0, 1);  // node type: group
    o.put(0, 1);  // level
    o.put(1, 2);  // entries used
    o.put(UNDEF, 8);
    o.put(UNDEF, 8);
    o.put(0, 8);
    const size_t at_child = o.pos();
    o.put(0, 8);
    o.put(name_off.empty() ? 0 : name_off.back(), 8);
    o.zeros(BTREE_NODE - (o.pos() - btree));

    // symbol table node: one entry per dataset (header addresses patched)
    o.align8();
    const size_t snod = o.pos();
    o.bytes("SNOD", 4);
    o.put(1, 1);  // version
    o.put(0, 1);
    o.put(ds.size(), 2);
    std::vector<size_t> at_entry_oh;
    for (size_t k = 0; k < ds.size(); ++k) {
        o.put(name_off[k], 8);
        at_entry_oh.push_back(o.pos());
        o.put(0, 8);
        o.put(0, 4);  // no cached data
        o.put(0, 4);
        o.zeros(16);
    }
    o.zeros(SNOD_NODE - (o.pos() - snod));

    // dataset object headers (data addresses patched once the data is placed)
    std::vector<size_t> at_data_addr;
    for (size_t k = 0; k < ds.size(); ++k) {
        const Dataset &d = ds[k];
        o.align8();
        o.patch(at_entry_oh[k], o.pos(), 8);
        Out space;  // dataspace, version 1
        space.put(1, 1);
        space.put(d.dims.size(), 1);
        space.put(0, 1);  // no maximum dimensions
        space.zeros(5);
        for (uint64_t n : d.dims) space.put(n, 8);
        Out type;
        if (d.integer) {
            type.put(0x10, 1);  // version 1, class 0 (fixed point)
            type.put(0x08, 1);  // little endian, signed
            type.put(0, 2);
            type.put(8, 4);     // size
            type.put(0, 2);     // bit offset
            type.put(64, 2);    // bit precision
        } else {
            type.put(0x11, 1);  // version 1, class 1 (floating point)
            type.put(0x20, 1);  // little endian, implied leading mantissa bit
            type.put(63, 1);    // sign bit location
            type.put(0, 1);
            type.put(8, 4);     // size
            type.put(0, 2);     // bit offset
            type.put(64, 2);    // bit precision
            type.put(52, 1);    // exponent location
            type.put(11, 1);    // exponent size
            type.put(0, 1);     // mantissa location
            type.put(52, 1);    // mantissa size
            type.put(1023, 4);  // exponent bias
        }
        Out layout;  // data layout, version 3, contiguous
        layout.put(3, 1);
        layout.put(1, 1);
        layout.put(0, 8);  // address (patched)
        layout.put(d.data.size(), 8);
        const size_t oh = o.pos();
        object_header(o, {{0x0001, space}, {0x0003, type}, {0x0008, layout}});
        at_data_addr.push_back(oh + 16 + (8 + pad8(space.b.size())) + (8 + pad8(type.b.size())) + 8 + 2);
    }
    // raw data
    for (size_t k = 0; k < ds.size(); ++k) {
        o.align8();
        o.patch(at_data_addr[k], o.pos(), 8);
        o.bytes(ds[k].data.data(), ds[k].data.size());
    }

    o.patch(at_root_oh, root_oh, 8);
    o.patch(at_root_bt, btree, 8);
    o.patch(at_root_heap, heap_hdr, 8);
    o.patch(at_msg_data + stab_bt, btree, 8);
    o.patch(at_msg_data + stab_heap, heap_hdr, 8);
    o.patch(at_child, snod, 8);
    o.patch(at_eof, o.pos(), 8);

    FILE *fp = std::fopen(path, "wb");
    if (!fp) throw LbmError(LBM_ERR_INVALID, std::string("cannot create HDF5 file ") + path);
    const size_t w = std::fwrite(o.b.data(), 1, o.b.size(), fp);
    const int c = std::fclose(fp);
    if (w != o.b.size() || c != 0) throw LbmError(LBM_ERR_INVALID, std::string("cannot write HDF5 file ") + path);
}

}  // namespace

void hdf5_write_fields(const char *path, int Nx, int Ny, const double *rho, const double *ux, const double *uy,
                       const double *T, double t, double gamma, double R, double T_ref, double rho_ref,
                       const double *dx, int ndx, const double *dy, int ndy, const double *f, const double *h)
{
    if (!path || Nx < 1 || Ny < 1 || !rho || !ux || !uy || !T || !dx || !dy || ndx < 1 || ndy < 1)
        throw LbmError(LBM_ERR_INVALID, "bad argument");
    const uint64_t X = (uint64_t)Nx, Y = (uint64_t)Ny;
    const size_t n = (size_t)Nx * Ny;
    std::vector<Dataset> ds;
    ds.push_back(doubles("rho", {X, Y}, rho, n));
    ds.push_back(doubles("T", {X, Y}, T, n));
    ds.push_back(doubles("ux", {X, Y}, ux, n));
    ds.push_back(doubles("uy", {X, Y}, uy, n));
    ds.push_back(scalar("t", t));
    ds.push_back(scalar("gamma", gamma));
    ds.push_back(scalar("R", R));
    ds.push_back(scalar("T_ref", T_ref));
    ds.push_back(scalar("rho_ref", rho_ref));
    ds.push_back(ndx == 1 ? scalar("dx", dx[0]) : doubles("dx", {(uint64_t)ndx}, dx, ndx));
    ds.push_back(ndy == 1 ? scalar("dy", dy[0]) : doubles("dy", {(uint64_t)ndy}, dy, ndy));
    ds.push_back(integer("Nx", Nx));
    ds.push_back(integer("Ny", Ny));
    if (f && h) {
        ds.push_back(doubles("f", {X, Y, (uint64_t)NDIR}, f, n * NDIR));
        ds.push_back(doubles("h", {X, Y, (uint64_t)NDIR}, h, n * NDIR));
    }
    write_file(path, std::move(ds));
}

}  // namespace uqlbm

using namespace uqlbm;

extern "C" {

LBM_API lbm_status lbm_hdf5_write_fields(const char *path, int Nx, int Ny, const double *rho, const double *ux,
                                         const double *uy, const double *T, double t, double gamma, double R,
                                         double T_ref, double rho_ref, const double *dx, int ndx, const double *dy,
                                         int ndy, const double *f, const double *h)
{
    try {
        hdf5_write_fields(path, Nx, Ny, rho, ux, uy, T, t, gamma, R, T_ref, rho_ref, dx, ndx, dy, ndy, f, h);
        return LBM_OK;
    } catch (const LbmError &e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc &) {
        g_last_error = "host allocation failed";
        return LBM_ERR_NOMEM;
    }
}

}  // extern "C"
