// fm_vti.cpp -- VTK ImageData (.vti) geometry reader and field writer (host code).
//
// fm_vti_read follows readVTI (include/vti/VTIReader.hpp:35-160): the
// dimensions come from WholeExtent (else Extent) "x0 x1 y0 y1 z0 z1"; the
// first <DataArray> holds Nx*Ny*Nz scalars or 3*Nx*Ny*Nz vector components
// (magnitude); mask = value > threshold; any other count keeps the first
// min(count, N) values (with the reference's warnings on stderr).  Beyond the
// reference's ASCII DataArray it reads format="binary" (base64, UInt32 or
// UInt64 block header) and format="appended" (raw or base64 AppendedData)
// arrays of every VTK scalar type, uncompressed, and returns the values
// themselves for continuous fields (a solid fraction n_s).  ASCII numbers are
// parsed with std::from_chars (no stream extraction per value).
#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fm.h"

namespace fm_internal {
int set_error(int code, const std::string& msg);
}

namespace {

int err(int code, const std::string& m) { return fm_internal::set_error(code, m); }

bool slurp(const char* path, std::string& out)
{
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    out.resize(sz > 0 ? (size_t)sz : 0);
    const size_t got = sz > 0 ? std::fread(&out[0], 1, (size_t)sz, f) : 0;
    std::fclose(f);
    out.resize(got);
    return true;
}

// value of name="..." inside [from, to)
std::string attr(const std::string& s, size_t from, size_t to, const char* name)
{
    const std::string pat = std::string(" ") + name + "=\"";
    size_t p = s.find(pat, from);
    if (p == std::string::npos || p >= to) {
        // attribute directly after a tab or newline
        for (const char* sep : {"\t", "\n", "\r"}) {
            const std::string p2 = std::string(sep) + name + "=\"";
            p = s.find(p2, from);
            if (p != std::string::npos && p < to) break;
        }
        if (p == std::string::npos || p >= to) return {};
    }
    p = s.find('"', p) + 1;
    const size_t e = s.find('"', p);
    if (e == std::string::npos) return {};
    return s.substr(p, e - p);
}

// the reference's findAttribute: first occurrence of name="..." anywhere
std::string attr_anywhere(const std::string& s, const char* name)
{
    const std::string pat = std::string(name) + "=\"";
    size_t p = s.find(pat);
    if (p == std::string::npos) return {};
    p += pat.size();
    const size_t e = s.find('"', p);
    if (e == std::string::npos) return {};
    return s.substr(p, e - p);
}

int b64val(unsigned char c)
{
    if (c >= 'A' && c <= 'Z') return c - 'A';
    if (c >= 'a' && c <= 'z') return c - 'a' + 26;
    if (c >= '0' && c <= '9') return c - '0' + 52;
    if (c == '+') return 62;
    if (c == '/') return 63;
    return -1;
}

// decode base64 (whitespace skipped; '=' ends a quantum)
std::vector<unsigned char> b64decode(const char* p, const char* e)
{
    std::vector<unsigned char> out;
    out.reserve((size_t)(e - p) * 3 / 4);
    uint32_t acc = 0;
    int bits = 0;
    for (; p < e; ++p) {
        const int v = b64val((unsigned char)*p);
        if (v < 0) continue;
        acc = (acc << 6) | (uint32_t)v;
        bits += 6;
        if (bits >= 8) {
            bits -= 8;
            out.push_back((unsigned char)((acc >> bits) & 0xFF));
        }
    }
    return out;
}

int type_size(const std::string& t)
{
    if (t == "Float32" || t == "Int32" || t == "UInt32") return 4;
    if (t == "Float64" || t == "Int64" || t == "UInt64") return 8;
    if (t == "Int16" || t == "UInt16") return 2;
    if (t == "Int8" || t == "UInt8") return 1;
    return 0;
}

double elem(const unsigned char* p, const std::string& t)
{
    if (t == "Float32") { float v; std::memcpy(&v, p, 4); return v; }
    if (t == "Float64") { double v; std::memcpy(&v, p, 8); return v; }
    if (t == "Int32") { int32_t v; std::memcpy(&v, p, 4); return v; }
    if (t == "UInt32") { uint32_t v; std::memcpy(&v, p, 4); return v; }
    if (t == "Int64") { int64_t v; std::memcpy(&v, p, 8); return (double)v; }
    if (t == "UInt64") { uint64_t v; std::memcpy(&v, p, 8); return (double)v; }
    if (t == "Int16") { int16_t v; std::memcpy(&v, p, 2); return v; }
    if (t == "UInt16") { uint16_t v; std::memcpy(&v, p, 2); return v; }
    if (t == "Int8") return (double)(int8_t)p[0];
    return (double)p[0];
}

// numbers of an ASCII DataArray body, as `stream >> double` reads them:
// stops at the first token that is not a number
void parse_ascii(const char* p, const char* e, std::vector<double>& vals)
{
    while (p < e) {
        while (p < e && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t' || *p == '\f' || *p == '\v')) ++p;
        if (p >= e) break;
        const char* q = (*p == '+') ? p + 1 : p;   // from_chars rejects a leading '+'
        double v;
        auto r = std::from_chars(q, e, v);
        if (r.ec != std::errc()) break;
        vals.push_back(v);
        p = r.ptr;
    }
}

struct Vti {
    int nx = 0, ny = 0, nz = 0;
    std::vector<double> vals;
};

int load(const char* path, Vti& out)
{
    std::string s;
    if (!path || !slurp(path, s)) return err(FM_ERR_ARG, std::string("[VTIReader]: Fatal, could not open File: ") + (path ? path : "(null)"));
    std::string ext = attr_anywhere(s, "WholeExtent");
    if (ext.empty()) ext = attr_anywhere(s, "Extent");
    if (ext.empty()) return err(FM_ERR_ARG, "[VTIReader]: Fatal, no Extent/WholeExtent found in VTI File!");
    long long e6[6];
    {
        const char* p = ext.c_str();
        const char* end = p + ext.size();
        for (int i = 0; i < 6; ++i) {
            while (p < end && (*p == ' ' || *p == '\t' || *p == '\n')) ++p;
            auto r = std::from_chars(p, end, e6[i]);
            if (r.ec != std::errc())
                return err(FM_ERR_ARG, "[VTIReader]: Fatal, could not parse Extent/WholeExtent! - " + ext);
            p = r.ptr;
        }
    }
    out.nx = (int)(e6[1] - e6[0] + 1);
    out.ny = (int)(e6[3] - e6[2] + 1);
    out.nz = (int)(e6[5] - e6[4] + 1);
    const size_t da = s.find("<DataArray");
    if (da == std::string::npos) return err(FM_ERR_ARG, "[VTIReader]: Fatal, no <DataArray> found in VTI File.");
    const size_t gt = s.find('>', da);
    if (gt == std::string::npos) return err(FM_ERR_ARG, "[VTIReader]: Fatal, invalid DataArray-Tag.");
    const std::string format = attr(s, da, gt, "format");
    const std::string type = attr(s, da, gt, "type");
    if (format.empty() || format == "ascii") {
        const size_t et = s.find("</DataArray>", gt);
        if (et == std::string::npos)
            return err(FM_ERR_ARG, "[VTIReader]: Fatal, could not found closing </DataArray>-Tag!");
        parse_ascii(s.data() + gt + 1, s.data() + et, out.vals);
    } else {
        if (attr_anywhere(s, "compressor").size())
            return err(FM_ERR_UNSUPPORTED, "[VTIReader]: compressed DataArray (compressor=...) is not supported");
        const int ts = type_size(type);
        if (!ts) return err(FM_ERR_UNSUPPORTED, "[VTIReader]: unsupported DataArray type " + type);
        const bool hdr64 = attr_anywhere(s, "header_type") == "UInt64";
        const size_t hb = hdr64 ? 8 : 4;
        std::vector<unsigned char> raw;
        if (format == "binary") {
            const size_t et = s.find("</DataArray>", gt);
            if (et == std::string::npos)
                return err(FM_ERR_ARG, "[VTIReader]: Fatal, could not found closing </DataArray>-Tag!");
            raw = b64decode(s.data() + gt + 1, s.data() + et);
        } else if (format == "appended") {
            const size_t ad = s.find("<AppendedData");
            if (ad == std::string::npos) return err(FM_ERR_ARG, "[VTIReader]: appended DataArray without <AppendedData>");
            const size_t agt = s.find('>', ad);
            const std::string enc = attr(s, ad, agt, "encoding");
            const size_t us = s.find('_', agt);
            if (us == std::string::npos) return err(FM_ERR_ARG, "[VTIReader]: <AppendedData> without '_' marker");
            const std::string off_s = attr(s, da, gt, "offset");
            const size_t off = off_s.empty() ? 0 : (size_t)std::strtoull(off_s.c_str(), nullptr, 10);
            if (enc == "base64") {
                const size_t end = s.find("</AppendedData>", us);
                raw = b64decode(s.data() + us + 1 + off, s.data() + (end == std::string::npos ? s.size() : end));
            } else {
                const size_t base = us + 1 + off;
                if (base + hb > s.size()) return err(FM_ERR_ARG, "[VTIReader]: appended data truncated");
                uint64_t nbytes = 0;
                std::memcpy(&nbytes, s.data() + base, hb);
                if (base + hb + nbytes > s.size()) return err(FM_ERR_ARG, "[VTIReader]: appended data truncated");
                raw.assign((const unsigned char*)s.data() + base, (const unsigned char*)s.data() + base + hb + nbytes);
            }
        } else {
            return err(FM_ERR_UNSUPPORTED, "[VTIReader]: unsupported DataArray format " + format);
        }
        if (raw.size() < hb) return err(FM_ERR_ARG, "[VTIReader]: binary DataArray without its size header");
        uint64_t nbytes = 0;
        std::memcpy(&nbytes, raw.data(), hb);
        nbytes = std::min<uint64_t>(nbytes, raw.size() - hb);
        const size_t count = (size_t)(nbytes / (uint64_t)ts);
        out.vals.resize(count);
        for (size_t i = 0; i < count; ++i) out.vals[i] = elem(raw.data() + hb + i * (size_t)ts, type);
    }
    if (out.vals.empty()) return err(FM_ERR_ARG, "[VTIReader]: Fatal, DataArray does not contain numerical values!");
    return FM_OK;
}

}  // namespace

extern "C" {

int fm_vti_info(const char* path, int* nx, int* ny, int* nz, long long* nvalues)
{
    Vti v;
    int rc = load(path, v);
    if (rc) return rc;
    if (nx) *nx = v.nx;
    if (ny) *ny = v.ny;
    if (nz) *nz = v.nz;
    if (nvalues) *nvalues = (long long)v.vals.size();
    return FM_OK;
}

int fm_vti_read(const char* path, double threshold, uint8_t* mask, double* values, size_t n)
{
    Vti v;
    int rc = load(path, v);
    if (rc) return rc;
    const size_t N = (size_t)v.nx * (size_t)v.ny * (size_t)v.nz;
    if (n != N) return err(FM_ERR_ARG, "fm_vti_read: output size " + std::to_string(n) + " != Nx*Ny*Nz " + std::to_string(N));
    const size_t nv = v.vals.size();
    std::vector<double> s(N, 0.0);
    if (nv == N) {
        s = v.vals;
    } else if (nv == 3 * N) {
        std::fprintf(stderr, "[VTIReader]: The DataArray seems to contain 3 Components per Cell - RGB?\n");
        for (size_t i = 0; i < N; ++i) {
            const double x = v.vals[3 * i], y = v.vals[3 * i + 1], z = v.vals[3 * i + 2];
            s[i] = std::sqrt(x * x + y * y + z * z);
        }
    } else {
        std::fprintf(stderr,
                     "[VTIReader]: Warning: Number of values (%zu) does not fit to Nx*Ny*Nz (%zu) or 3*Nx*Ny*Nz. "
                     "Mask will be cut and there might be problems...\n",
                     nv, N);
        for (size_t i = 0; i < std::min(nv, N); ++i) s[i] = v.vals[i];
    }
    const size_t valid = (nv == N || nv == 3 * N) ? N : std::min(nv, N);
    if (mask)
        for (size_t i = 0; i < N; ++i) mask[i] = (i < valid && s[i] > threshold) ? 1u : 0u;
    if (values) std::memcpy(values, s.data(), N * sizeof(double));
    return FM_OK;
}

int fm_vti_write(const char* path, int nx, int ny, int nz, const double* values, int components, const char* name,
                 int binary)
{
    if (!path || !values || nx <= 0 || ny <= 0 || nz <= 0 || (components != 1 && components != 3))
        return err(FM_ERR_ARG, "fm_vti_write: bad arguments");
    FILE* f = std::fopen(path, "wb");
    if (!f) return err(FM_ERR_ARG, std::string("fm_vti_write: could not open ") + path);
    const size_t N = (size_t)nx * ny * nz * (size_t)components;
    const char* nm = name ? name : "field";
    std::fprintf(f, "<?xml version=\"1.0\"?>\n<VTKFile type=\"ImageData\" version=\"1.0\" byte_order=\"LittleEndian\" "
                    "header_type=\"UInt64\">\n  <ImageData WholeExtent=\"0 %d 0 %d 0 %d\" Origin=\"0 0 0\" "
                    "Spacing=\"1 1 1\">\n    <Piece Extent=\"0 %d 0 %d 0 %d\">\n      <CellData Scalars=\"%s\">\n",
                 nx - 1, ny - 1, nz - 1, nx - 1, ny - 1, nz - 1, nm);
    if (binary) {
        std::fprintf(f, "        <DataArray type=\"Float64\" Name=\"%s\" NumberOfComponents=\"%d\" format=\"appended\" "
                        "offset=\"0\"/>\n      </CellData>\n    </Piece>\n  </ImageData>\n  <AppendedData "
                        "encoding=\"raw\">\n   _",
                     nm, components);
        const uint64_t nb = (uint64_t)N * 8;
        std::fwrite(&nb, 8, 1, f);
        std::fwrite(values, 8, N, f);
        std::fprintf(f, "\n  </AppendedData>\n</VTKFile>\n");
    } else {
        std::fprintf(f, "        <DataArray type=\"Float64\" Name=\"%s\" NumberOfComponents=\"%d\" format=\"ascii\">\n",
                     nm, components);
        char buf[64];
        for (size_t i = 0; i < N; ++i) {
            auto r = std::to_chars(buf, buf + sizeof(buf), values[i]);
            *r.ptr = (i % 8 == 7 || i + 1 == N) ? '\n' : ' ';
            std::fwrite(buf, 1, (size_t)(r.ptr - buf) + 1, f);
        }
        std::fprintf(f, "        </DataArray>\n      </CellData>\n    </Piece>\n  </ImageData>\n</VTKFile>\n");
    }
    const bool ok = std::fclose(f) == 0;
    return ok ? FM_OK : err(FM_ERR_ARG, std::string("fm_vti_write: write failed ") + path);
}

}  // extern "C"
