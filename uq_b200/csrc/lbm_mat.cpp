// MATLAB Level-5 MAT files at the boundary: the reference's input files
// (read by cpuLBM::loadInput, CODE/C++/VS2010/simLB/simLB/cpuLBM.cpp:46-281)
// and its output files (cpuLBM::createMAT, cpuLBM.cpp:467-745).
//
// The reader follows the published Level-5 layout: a 128-byte header, then
// data elements (8-byte tag: type, byte count; payload padded to 8 bytes,
// or the 4-byte "small element" form), numeric arrays as miMATRIX elements
// (array flags, dimensions, name, real part), and whole variables
// zlib-compressed inside miCOMPRESSED elements.  Every numeric class is
// converted to double, which is how loadInput reads each variable (through
// mxGetPr).  The writer emits uncompressed double arrays.
#include "lbm_mat.h"

#include "lbm_host.h"

#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace uqlbm {
namespace {

enum : uint32_t {
    miINT8 = 1, miUINT8 = 2, miINT16 = 3, miUINT16 = 4, miINT32 = 5, miUINT32 = 6, miSINGLE = 7, miDOUBLE = 9,
    miINT64 = 12, miUINT64 = 13, miMATRIX = 14, miCOMPRESSED = 15, miUTF8 = 16
};
enum : uint32_t { mxCHAR = 4, mxSPARSE = 5, mxDOUBLE = 6, mxUINT64 = 15 };

struct Reader {
    const uint8_t *p;
    size_t n, pos = 0;
    bool swap;
    uint32_t u32(size_t at) const
    {
        uint32_t v;
        std::memcpy(&v, p + at, 4);
        return swap ? __builtin_bswap32(v) : v;
    }
};

// one data element: type, payload pointer and length, and the offset of
// the next element
struct Element {
    uint32_t type;
    const uint8_t *data;
    size_t len, next;
};

bool read_element(const Reader &r, size_t at, Element &e)
{
    if (at + 8 > r.n) return false;
    const uint32_t w0 = r.u32(at);
    if (w0 >> 16) {  // small data element: 2-byte count, 2-byte type, 4 bytes of data
        e.type = w0 & 0xffff;
        e.len = w0 >> 16;
        e.data = r.p + at + 4;
        e.next = at + 8;
        return e.len <= 4;
    }
    e.type = w0;
    e.len = r.u32(at + 4);
    e.data = r.p + at + 8;
    if (at + 8 + e.len > r.n) return false;
    // compressed variables are not padded; everything else ends on 8 bytes
    e.next = at + 8 + (e.type == miCOMPRESSED ? e.len : (e.len + 7) / 8 * 8);
    return true;
}

template <class T>
T load_as(const uint8_t *q, bool swap)
{
    T v;
    std::memcpy(&v, q, sizeof(T));
    if (swap && sizeof(T) > 1) {
        uint8_t b[sizeof(T)];
        std::memcpy(b, &v, sizeof(T));
        for (size_t i = 0; i < sizeof(T) / 2; ++i) std::swap(b[i], b[sizeof(T) - 1 - i]);
        std::memcpy(&v, b, sizeof(T));
    }
    return v;
}

// numeric payload of any storage type -> doubles
bool numeric_to_double(uint32_t type, const uint8_t *q, size_t len, bool swap, std::vector<double> &out)
{
    size_t es = 0;
    switch (type) {
    case miINT8: case miUINT8: es = 1; break;
    case miINT16: case miUINT16: es = 2; break;
    case miINT32: case miUINT32: case miSINGLE: es = 4; break;
    case miDOUBLE: case miINT64: case miUINT64: es = 8; break;
    default: return false;
    }
    const size_t k = len / es;
    out.resize(k);
    for (size_t i = 0; i < k; ++i) {
        const uint8_t *e = q + i * es;
        switch (type) {
        case miINT8: out[i] = (double)load_as<int8_t>(e, swap); break;
        case miUINT8: out[i] = (double)load_as<uint8_t>(e, swap); break;
        case miINT16: out[i] = (double)load_as<int16_t>(e, swap); break;
        case miUINT16: out[i] = (double)load_as<uint16_t>(e, swap); break;
        case miINT32: out[i] = (double)load_as<int32_t>(e, swap); break;
        case miUINT32: out[i] = (double)load_as<uint32_t>(e, swap); break;
        case miSINGLE: out[i] = (double)load_as<float>(e, swap); break;
        case miDOUBLE: out[i] = load_as<double>(e, swap); break;
        case miINT64: out[i] = (double)load_as<int64_t>(e, swap); break;
        case miUINT64: out[i] = (double)load_as<uint64_t>(e, swap); break;
        }
    }
    return true;
}

struct Variable {
    std::vector<size_t> dims;
    std::vector<double> data;  // column-major, as stored
};

// parse one miMATRIX payload; non-numeric classes are skipped (ok = false)
bool parse_matrix(const Reader &r, const uint8_t *q, size_t len, std::string &name, Variable &v)
{
    Reader sub{q, len, 0, r.swap};
    Element flags, dims, nm, real;
    if (!read_element(sub, 0, flags) || flags.type != miUINT32 || flags.len < 8) return false;
    const uint32_t cls = sub.u32((size_t)(flags.data - q)) & 0xff;
    if (!read_element(sub, flags.next, dims) || dims.type != miINT32) return false;
    v.dims.clear();
    for (size_t i = 0; i + 4 <= dims.len; i += 4) {
        const int32_t d = load_as<int32_t>(dims.data + i, r.swap);
        if (d < 0) throw LbmError(LBM_ERR_INVALID, "MAT variable with a negative dimension");
        v.dims.push_back((size_t)d);
    }
    if (!read_element(sub, dims.next, nm) || (nm.type != miINT8 && nm.type != miUTF8)) return false;
    name.assign(reinterpret_cast<const char *>(nm.data), nm.len);
    if (cls < mxDOUBLE || cls > mxUINT64 || cls == mxSPARSE || cls == mxCHAR) return false;
    if (!read_element(sub, nm.next, real)) return false;
    size_t count = 1;
    for (size_t d : v.dims)
        if (__builtin_mul_overflow(count, d, &count))
            throw LbmError(LBM_ERR_INVALID, "MAT variable whose element count overflows");
    if (!numeric_to_double(real.type, real.data, real.len, r.swap, v.data) || v.data.size() != count) return false;
    return true;
}

bool inflate_all(const uint8_t *q, size_t len, std::vector<uint8_t> &out)
{
    z_stream zs{};
    if (inflateInit(&zs) != Z_OK) return false;
    zs.next_in = const_cast<Bytef *>(q);
    zs.avail_in = (uInt)len;
    out.assign(std::max<size_t>(len * 8, 4096), 0);
    int rc;
    do {
        if (zs.total_out == out.size()) out.resize(out.size() * 2);
        zs.next_out = out.data() + zs.total_out;
        zs.avail_out = (uInt)(out.size() - zs.total_out);
        rc = inflate(&zs, Z_NO_FLUSH);
    } while (rc == Z_OK);
    out.resize(zs.total_out);
    inflateEnd(&zs);
    return rc == Z_STREAM_END;
}

std::map<std::string, Variable> read_mat(const char *path)
{
    std::unique_ptr<FILE, int (*)(FILE *)> f(std::fopen(path, "rb"), std::fclose);
    if (!f) throw LbmError(LBM_ERR_INVALID, std::string("cannot open MAT file ") + path);
    std::vector<uint8_t> buf;
    uint8_t chunk[1 << 16];
    size_t k;
    while ((k = std::fread(chunk, 1, sizeof(chunk), f.get())) > 0) buf.insert(buf.end(), chunk, chunk + k);
    if (buf.size() < 128) throw LbmError(LBM_ERR_INVALID, "not a Level-5 MAT file (short header)");
    bool swap;
    if (buf[126] == 'I' && buf[127] == 'M') swap = false;
    else if (buf[126] == 'M' && buf[127] == 'I') swap = true;
    else throw LbmError(LBM_ERR_INVALID, "not a Level-5 MAT file (no endian indicator)");
    Reader r{buf.data(), buf.size(), 128, swap};
    std::map<std::string, Variable> vars;
    size_t at = 128;
    while (at + 8 <= r.n) {
        Element e;
        if (!read_element(r, at, e)) throw LbmError(LBM_ERR_INVALID, "truncated MAT data element");
        std::string name;
        Variable v;
        if (e.type == miMATRIX) {
            if (parse_matrix(r, e.data, e.len, name, v)) vars[name] = std::move(v);
        } else if (e.type == miCOMPRESSED) {
            std::vector<uint8_t> raw;
            if (!inflate_all(e.data, e.len, raw)) throw LbmError(LBM_ERR_INVALID, "corrupt compressed MAT variable");
            Reader ir{raw.data(), raw.size(), 0, swap};
            Element inner;
            if (read_element(ir, 0, inner) && inner.type == miMATRIX &&
                parse_matrix(ir, inner.data, inner.len, name, v))
                vars[name] = std::move(v);
        }
        at = e.next;
    }
    return vars;
}

// ----------------------------------------------------------------- writer
void put_u32(std::vector<uint8_t> &b, uint32_t v)
{
    uint8_t q[4];
    std::memcpy(q, &v, 4);
    b.insert(b.end(), q, q + 4);
}

void pad8(std::vector<uint8_t> &b)
{
    while (b.size() % 8) b.push_back(0);
}

void put_double_array(std::vector<uint8_t> &out, const char *name, const std::vector<uint32_t> &dims, const double *d)
{
    size_t count = 1;
    for (uint32_t x : dims) count *= x;
    std::vector<uint8_t> m;
    put_u32(m, miUINT32);  // array flags
    put_u32(m, 8);
    put_u32(m, mxDOUBLE);
    put_u32(m, 0);
    put_u32(m, miINT32);  // dimensions
    put_u32(m, (uint32_t)(4 * dims.size()));
    for (uint32_t x : dims) put_u32(m, x);
    pad8(m);
    const size_t nl = std::strlen(name);
    put_u32(m, miINT8);  // name
    put_u32(m, (uint32_t)nl);
    m.insert(m.end(), name, name + nl);
    pad8(m);
    put_u32(m, miDOUBLE);  // real part
    put_u32(m, (uint32_t)(8 * count));
    const uint8_t *q = reinterpret_cast<const uint8_t *>(d);
    m.insert(m.end(), q, q + 8 * count);
    pad8(m);
    put_u32(out, miMATRIX);
    put_u32(out, (uint32_t)m.size());
    out.insert(out.end(), m.begin(), m.end());
}

}  // namespace

void mat_read_case(const char *path, MatCase &c)
{
    const auto vars = read_mat(path);
    auto scalar = [&](const char *n, double dflt) {
        auto it = vars.find(n);
        return (it == vars.end() || it->second.data.empty()) ? dflt : it->second.data[0];
    };
    auto vec = [&](const char *n) -> const Variable & {
        auto it = vars.find(n);
        if (it == vars.end() || it->second.data.empty())
            throw LbmError(LBM_ERR_INVALID, std::string("MAT input lacks the variable ") + n);
        return it->second;
    };
    lbm_config &g = c.cfg;
    g = lbm_config{};
    // cpuLBM.cpp:113-199 (scalar variables, same names)
    g.RKMETHOD = (int)scalar("RKMETHOD", 0);
    g.FMETHOD = (int)scalar("FMETHOD", 0);
    g.CFL = scalar("CFL", 0);
    g.dtau = scalar("dtau", 0);
    g.tt_tref = scalar("tt_tref", 0);
    g.tt_time = scalar("tt_time", 0);
    g.steps = (int)scalar("steps", 0);
    g.tol = scalar("tol", 0);
    g.periodicX = (int)scalar("periodicX", 0);
    g.periodicY = (int)scalar("periodicY", 0);
    g.mirrorNorth = (int)scalar("mirrorNorth", 0);
    g.mirrorSouth = (int)scalar("mirrorSouth", 0);
    g.mirrorEast = (int)scalar("mirrorEast", 0);
    g.mirrorWest = (int)scalar("mirrorWest", 0);
    g.gamma = scalar("gamma", 0);
    g.R = scalar("R", 0);
    g.mu = scalar("mu", 0);
    g.Pr = scalar("Pr", 0);
    g.dx = scalar("dx", 0);
    g.dy = scalar("dy", 0);
    g.Lx = scalar("Lx", 0);
    g.Ly = scalar("Ly", 0);
    g.rho_ref = scalar("rho_ref", 0);
    g.p_ref = scalar("p_ref", 0);
    g.T_ref = scalar("T_ref", 0);
    g.Tc_Tref = scalar("Tc_Tref", 0);
    // optional: the OpenCL generator's viscosity law (absent: constant mu,
    // as in loadInput)
    g.mu_model = (int)scalar("mu_model", 0);
    g.upsilon = scalar("upsilon", 0);
    g.S_v = scalar("S_v", 0);
    // property tables (cpuLBM.cpp:201-250): max(dims) entries each
    const int np = (int)scalar("numProps", 0);
    auto table = [&](const char *n, std::vector<double> &dst) {
        const Variable &v = vec(n);
        dst = v.data;
        if ((int)dst.size() < np) throw LbmError(LBM_ERR_INVALID, std::string("MAT table too short: ") + n);
    };
    table("density", c.density);
    table("pressure", c.pressure);
    table("temp", c.temp);
    table("velocityX", c.velocityX);
    table("velocityY", c.velocityY);
    std::vector<double> ct;
    table("cellType", ct);
    c.cellType.assign(ct.begin(), ct.end());
    // bndArray (cpuLBM.cpp:252-264): Nx = dims[1], Ny = dims[0], y flipped
    const Variable &b = vec("bndArray");
    if (b.dims.size() != 2) throw LbmError(LBM_ERR_INVALID, "bndArray must be two-dimensional");
    const int Ny = (int)b.dims[0], Nx = (int)b.dims[1];
    c.bnd.resize((size_t)Nx * Ny);
    for (int y = 0; y < Ny; ++y)
        for (int x = 0; x < Nx; ++x) c.bnd[(size_t)x * Ny + y] = (int)b.data[(size_t)x * Ny + (Ny - 1 - y)];
    lbm_init &in = c.init;
    in = lbm_init{};
    in.Nx = Nx;
    in.Ny = Ny;
    in.numProps = np;
    in.bndArray = c.bnd.data();
    in.cellType = c.cellType.data();
    in.density = c.density.data();
    in.pressure = c.pressure.data();
    in.temp = c.temp.data();
    in.velocityX = c.velocityX.data();
    in.velocityY = c.velocityY.data();
}

void mat_read_dist(const char *path, int Nx, int Ny, double *f, double *h, double *t)
{
    const auto vars = read_mat(path);
    const size_t n = (size_t)Nx * Ny * 13;
    const char *names[2] = {"f", "h"};
    double *dst[2] = {f, h};
    for (int k = 0; k < 2; ++k) {
        auto it = vars.find(names[k]);
        if (it == vars.end()) throw LbmError(LBM_ERR_INVALID, std::string("MAT checkpoint lacks ") + names[k]);
        const Variable &v = it->second;
        if (v.dims.size() != 3 || v.dims[0] != 13 || v.dims[1] != (size_t)Ny || v.dims[2] != (size_t)Nx)
            throw LbmError(LBM_ERR_INVALID, std::string("MAT checkpoint: ") + names[k] + " is not 13 x Ny x Nx");
        if (dst[k]) std::copy(v.data.begin(), v.data.begin() + n, dst[k]);  // column-major = [(x*Ny + y)*13 + i]
    }
    auto it = vars.find("t");
    if (t) *t = (it == vars.end() || it->second.data.empty()) ? 0.0 : it->second.data[0];
}

void mat_write_fields(const char *path, int Nx, int Ny, const double *rho, const double *ux, const double *uy,
                      const double *p, const double *T, double t, double dx, double dy, const double *f,
                      const double *h, const double *ex, const double *ey)
{
    if (!path || Nx < 1 || Ny < 1 || !rho || !ux || !uy || !p || !T)
        throw LbmError(LBM_ERR_INVALID, "MAT output needs a path and the five fields");
    std::vector<uint8_t> out(128, ' ');
    const char *text = "MATLAB 5.0 MAT-file, written by libuqlbm";
    std::memcpy(out.data(), text, std::strlen(text));
    std::memset(out.data() + 116, 0, 8);  // no subsystem data
    out[124] = 0x00;
    out[125] = 0x01;  // version 0x0100, stored little-endian
    out[126] = 'I';
    out[127] = 'M';
    // createMAT's order and shapes: fields {Ny, Nx} over [x*Ny + y] data,
    // distributions {13, Ny, Nx} over [(x*Ny + y)*13 + i]
    const std::vector<uint32_t> d2 = {(uint32_t)Ny, (uint32_t)Nx}, d1 = {1, 1};
    if (f && h && ex && ey) {
        const std::vector<uint32_t> d3 = {13, (uint32_t)Ny, (uint32_t)Nx}, de = {13, 1};
        put_double_array(out, "f", d3, f);
        put_double_array(out, "h", d3, h);
        put_double_array(out, "ex", de, ex);
        put_double_array(out, "ey", de, ey);
    }
    put_double_array(out, "rho", d2, rho);
    put_double_array(out, "ux", d2, ux);
    put_double_array(out, "uy", d2, uy);
    put_double_array(out, "p", d2, p);
    put_double_array(out, "T", d2, T);
    put_double_array(out, "t", d1, &t);
    put_double_array(out, "dx", d1, &dx);
    put_double_array(out, "dy", d1, &dy);
    std::unique_ptr<FILE, int (*)(FILE *)> fo(std::fopen(path, "wb"), std::fclose);
    if (!fo) throw LbmError(LBM_ERR_INVALID, std::string("cannot create MAT file ") + path);
    if (std::fwrite(out.data(), 1, out.size(), fo.get()) != out.size())
        throw LbmError(LBM_ERR_INVALID, std::string("short write to ") + path);
}

}  // namespace uqlbm

// ---------------------------------------------------------------- C ABI
using namespace uqlbm;

struct lbm_mat_case {
    MatCase c;
};

#define MAT_BEGIN try {
#define MAT_END                                          \
    }                                                    \
    catch (const LbmError &e)                            \
    {                                                    \
        g_last_error = e.what();                         \
        return e.code;                                   \
    }                                                    \
    catch (const std::bad_alloc &)                       \
    {                                                    \
        g_last_error = "host allocation failed";         \
        return LBM_ERR_NOMEM;                            \
    }                                                    \
    catch (const std::exception &e)                      \
    {                                                    \
        g_last_error = e.what();                         \
        return LBM_ERR_INVALID;                          \
    }

extern "C" {

LBM_API lbm_status lbm_mat_read_case(const char *path, lbm_mat_case **out)
{
    MAT_BEGIN
    if (!path || !out) throw LbmError(LBM_ERR_INVALID, "NULL argument");
    *out = nullptr;
    std::unique_ptr<lbm_mat_case> m(new lbm_mat_case);
    mat_read_case(path, m->c);
    *out = m.release();
    return LBM_OK;
    MAT_END
}

LBM_API lbm_status lbm_mat_case_get(const lbm_mat_case *c, lbm_config *cfg, lbm_init *init)
{
    MAT_BEGIN
    if (!c) throw LbmError(LBM_ERR_INVALID, "NULL case");
    if (cfg) *cfg = c->c.cfg;
    if (init) *init = c->c.init;
    return LBM_OK;
    MAT_END
}

LBM_API void lbm_mat_case_free(lbm_mat_case *c) { delete c; }

LBM_API lbm_status lbm_mat_read_dist(const char *path, int Nx, int Ny, double *f, double *h, double *t)
{
    MAT_BEGIN
    if (!path || Nx < 1 || Ny < 1) throw LbmError(LBM_ERR_INVALID, "bad argument");
    mat_read_dist(path, Nx, Ny, f, h, t);
    return LBM_OK;
    MAT_END
}

LBM_API lbm_status lbm_mat_write_fields(const char *path, int Nx, int Ny, const double *rho, const double *ux,
                                        const double *uy, const double *p, const double *T, double t, double dx,
                                        double dy, const double *f, const double *h, const double *ex,
                                        const double *ey)
{
    MAT_BEGIN
    mat_write_fields(path, Nx, Ny, rho, ux, uy, p, T, t, dx, dy, f, h, ex, ey);
    return LBM_OK;
    MAT_END
}

}  // extern "C"
