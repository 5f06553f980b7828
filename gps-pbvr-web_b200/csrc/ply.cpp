// 3DGS PLY loader: a C++ restatement of crates/gps-io/src/lib.rs (load_ply :260-338,
// parse_header :165-238, push_vertex :341-373, activated :84-96) followed by
// GpuGaussian::from_activated (crates/gps-render/src/gps.rs:41-49). ASCII and binary
// little-endian, SH degree 0..3, validation without aborting on bad input.
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/gpsb200.h"
#include "ply_layout.h"

namespace {

const size_t kMaxVertices = 200000000;  // gps-io lib.rs:14
const double kShC0 = 0.28209479177387814;

enum Scalar { I8, U8, I16, U16, I32, U32, F32, F64 };
struct Prop { std::string name; Scalar ty; size_t off; };

bool parse_scalar(const std::string& s, Scalar* out) {
    static const struct { const char* a; Scalar t; } tab[] = {
        {"char", I8}, {"int8", I8}, {"uchar", U8}, {"uint8", U8}, {"short", I16}, {"int16", I16},
        {"ushort", U16}, {"uint16", U16}, {"int", I32}, {"int32", I32}, {"uint", U32}, {"uint32", U32},
        {"float", F32}, {"float32", F32}, {"double", F64}, {"float64", F64}};
    for (auto& e : tab)
        if (s == e.a) { *out = e.t; return true; }
    return false;
}
size_t scalar_size(Scalar t) {
    switch (t) {
        case I8: case U8: return 1;
        case I16: case U16: return 2;
        case I32: case U32: case F32: return 4;
        default: return 8;
    }
}
double read_le(Scalar t, const uint8_t* b) {
    switch (t) {
        case I8: return (double)(int8_t)b[0];
        case U8: return (double)b[0];
        case I16: { int16_t v; memcpy(&v, b, 2); return v; }
        case U16: { uint16_t v; memcpy(&v, b, 2); return v; }
        case I32: { int32_t v; memcpy(&v, b, 4); return v; }
        case U32: { uint32_t v; memcpy(&v, b, 4); return v; }
        case F32: { float v; memcpy(&v, b, 4); return v; }
        default: { double v; memcpy(&v, b, 8); return v; }
    }
}

thread_local std::string g_err;
gpsb_status perr(const std::string& m) {
    g_err = m;
    return GPSB_ERR_PARSE;
}

struct Header {
    bool binary = false, has_format = false, has_vertex = false;
    size_t count = 0, stride = 0, data_start = 0;
    std::vector<Prop> props;
};

gpsb_status parse_header(const uint8_t* bytes, size_t len, Header* h) {
    const char* marker = "end_header";
    size_t ml = strlen(marker), pos = (size_t)-1;
    for (size_t i = 0; i + ml <= len; ++i)
        if (memcmp(bytes + i, marker, ml) == 0) { pos = i; break; }
    if (pos == (size_t)-1) return perr("bad PLY header: no end_header");
    size_t ds = pos + ml;
    if (ds < len && bytes[ds] == '\r') ++ds;
    if (ds < len && bytes[ds] == '\n') ++ds;
    else return perr("bad PLY header: end_header not followed by newline");
    h->data_start = ds;
    std::string text((const char*)bytes, pos);
    std::vector<std::string> lines;
    size_t s = 0;
    while (s <= text.size()) {
        size_t e = text.find('\n', s);
        if (e == std::string::npos) e = text.size();
        std::string l = text.substr(s, e - s);
        if (!l.empty() && l.back() == '\r') l.pop_back();
        lines.push_back(l);
        s = e + 1;
    }
    auto trim = [](std::string x) {
        size_t a = x.find_first_not_of(" \t"), b = x.find_last_not_of(" \t");
        return a == std::string::npos ? std::string() : x.substr(a, b - a + 1);
    };
    if (lines.empty() || trim(lines[0]) != "ply") { g_err = "not a PLY file"; return GPSB_ERR_PARSE; }
    bool in_vertex = false, other_before = false;
    size_t off = 0;
    for (size_t li = 1; li < lines.size(); ++li) {
        std::vector<std::string> t;
        {
            size_t a = 0;
            const std::string& L = lines[li];
            while (a < L.size()) {
                while (a < L.size() && (L[a] == ' ' || L[a] == '\t')) ++a;
                size_t b = a;
                while (b < L.size() && L[b] != ' ' && L[b] != '\t') ++b;
                if (b > a) t.push_back(L.substr(a, b - a));
                a = b;
            }
        }
        if (t.size() == 3 && t[0] == "format") {
            if (t[1] == "ascii") h->binary = false;
            else if (t[1] == "binary_little_endian") h->binary = true;
            else return perr("unsupported PLY format: " + t[1]);
            h->has_format = true;
        } else if (t.size() == 3 && t[0] == "element") {
            in_vertex = t[1] == "vertex";
            if (in_vertex) {
                char* end = nullptr;
                unsigned long long n = strtoull(t[2].c_str(), &end, 10);
                if (!end || *end || t[2].empty() || t[2][0] == '-') return perr("bad PLY header: vertex count");
                if (n > kMaxVertices) return perr("vertex count " + t[2] + " exceeds limit 200000000");
                h->count = (size_t)n;
                h->has_vertex = true;
            } else if (!h->has_vertex) {
                other_before = true;
            }
        } else if (t.size() >= 2 && t[0] == "property" && t[1] == "list") {
            if (in_vertex) return perr("unsupported PLY format: list property in vertex element");
        } else if (t.size() == 3 && t[0] == "property" && in_vertex) {
            Scalar ty;
            if (!parse_scalar(t[1], &ty)) return perr("bad PLY header: type " + t[1]);
            h->props.push_back({t[2], ty, off});
            off += scalar_size(ty);
        }
    }
    if (other_before) return perr("unsupported PLY format: element before vertex");
    if (!h->has_format) return perr("bad PLY header: no format line");
    if (!h->has_vertex) return perr("bad PLY header: no vertex element");
    h->stride = off;
    return GPSB_OK;
}

int find(const Header& h, const std::string& n) {
    for (size_t i = 0; i < h.props.size(); ++i)
        if (h.props[i].name == n) return (int)i;
    return -1;
}

}  // namespace

namespace gpsb {

// Header, required-property lookup and SH degree of gpsb_load_ply, shared with the GPU decoder.
gpsb_status ply_layout(const uint8_t* bytes, size_t len, PlyLayout* out) {
    Header h;
    gpsb_status s = parse_header(bytes, len, &h);
    if (s != GPSB_OK) return s;
    const char* req[] = {"x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0", "scale_1", "scale_2",
                         "rot_0", "rot_1", "rot_2", "rot_3"};
    out->nprop = 0;
    for (int k = 0; k < 14; ++k) {
        int p = find(h, req[k]);
        if (p < 0) return perr(std::string("missing required property '") + req[k] + "'");
        out->off[out->nprop] = (uint32_t)h.props[p].off;
        out->type[out->nprop++] = (uint8_t)h.props[p].ty;
    }
    int nrest = 0;
    while (find(h, "f_rest_" + std::to_string(nrest)) >= 0) ++nrest;
    if (nrest != 0 && nrest != 9 && nrest != 24 && nrest != 45)
        return perr(std::to_string(nrest) + " f_rest_* properties is not 9, 24 or 45");
    for (int r = 0; r < nrest; ++r) {
        int p = find(h, "f_rest_" + std::to_string(r));
        out->off[out->nprop] = (uint32_t)h.props[p].off;
        out->type[out->nprop++] = (uint8_t)h.props[p].ty;
    }
    out->degree = nrest == 0 ? 0 : nrest == 9 ? 1 : nrest == 24 ? 2 : 3;
    out->binary = h.binary;
    out->count = h.count;
    out->stride = h.stride;
    out->data_start = h.data_start;
    if (h.binary) {
        size_t body_len = len - h.data_start;
        if (h.stride && h.count > (size_t)-1 / h.stride) return perr("vertex count too large");
        if (body_len < h.count * h.stride) {
            char buf[160];
            snprintf(buf, sizeof buf, "file truncated: need %zu bytes of vertex data, have %zu", h.count * h.stride,
                     body_len);
            return perr(buf);
        }
    }
    return GPSB_OK;
}

gpsb_status ply_error(const char* msg) { return perr(msg); }

}  // namespace gpsb

extern "C" {

const char* gpsb_ply_last_error(void) { return g_err.c_str(); }

gpsb_status gpsb_load_ply(const uint8_t* bytes, size_t len, size_t* n_out, uint32_t* sh_degree_out, gpsb_gaussian* splats,
                          float* sh_rest) {
    if (!bytes || !n_out || !sh_degree_out) return GPSB_ERR_INVALID_ARGUMENT;
    Header h;
    gpsb_status s = parse_header(bytes, len, &h);
    if (s != GPSB_OK) return s;
    const char* req[] = {"x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0", "scale_1", "scale_2",
                         "rot_0", "rot_1", "rot_2", "rot_3"};
    int idx[14];
    for (int k = 0; k < 14; ++k) {
        idx[k] = find(h, req[k]);
        if (idx[k] < 0) return perr(std::string("missing required property '") + req[k] + "'");
    }
    std::vector<int> irest;
    for (;;) {
        int p = find(h, "f_rest_" + std::to_string(irest.size()));
        if (p < 0) break;
        irest.push_back(p);
    }
    uint32_t deg;
    switch (irest.size()) {
        case 0: deg = 0; break;
        case 9: deg = 1; break;
        case 24: deg = 2; break;
        case 45: deg = 3; break;
        default: return perr(std::to_string(irest.size()) + " f_rest_* properties is not 9, 24 or 45");
    }
    const size_t n = h.count, per_ch = deg ? (deg + 1) * (deg + 1) - 1 : 0;
    const uint8_t* body = bytes + h.data_start;
    size_t body_len = len - h.data_start;
    if (h.binary) {
        if (h.stride && n > (size_t)-1 / h.stride) return perr("vertex count too large");
        if (body_len < n * h.stride) {
            char buf[160];
            snprintf(buf, sizeof buf, "file truncated: need %zu bytes of vertex data, have %zu", n * h.stride, body_len);
            return perr(buf);
        }
    } else {
        size_t need = n * std::max<size_t>(h.props.size(), 1) * 2;
        if (body_len + 1 < need) return perr("file truncated");
    }
    *n_out = n;
    *sh_degree_out = deg;
    if (!splats) return GPSB_OK;  // size query
    const char* field_of[14] = {"position", "position", "position", "f_dc", "f_dc", "f_dc", "opacity", "scale", "scale",
                                "scale", "rot", "rot", "rot", "rot"};
    std::vector<double> vals(h.props.size());
    const char* cursor = (const char*)body;
    const char* endp = (const char*)body + body_len;
    for (size_t v = 0; v < n; ++v) {
        if (h.binary) {
            const uint8_t* rec = body + v * h.stride;
            for (size_t p = 0; p < h.props.size(); ++p) vals[p] = (double)(float)read_le(h.props[p].ty, rec + h.props[p].off);
        } else {
            // skip blank lines, then parse one line of values
            while (cursor < endp && (*cursor == '\n' || *cursor == '\r' || *cursor == ' ' || *cursor == '\t')) ++cursor;
            if (cursor >= endp) return perr("file truncated: vertex " + std::to_string(v));
            const char* eol = cursor;
            while (eol < endp && *eol != '\n') ++eol;
            std::string line(cursor, eol - cursor);
            cursor = eol;
            const char* c = line.c_str();
            for (size_t p = 0; p < h.props.size(); ++p) {
                char* e = nullptr;
                while (*c == ' ' || *c == '\t') ++c;
                if (!*c) return perr("ASCII parse error at vertex " + std::to_string(v) + ": too few values");
                float x = strtof(c, &e);
                if (e == c) return perr("ASCII parse error at vertex " + std::to_string(v));
                vals[p] = (double)x;
                c = e;
            }
        }
        float f[14];
        for (int k = 0; k < 14; ++k) {
            f[k] = (float)vals[idx[k]];
            if (!std::isfinite(f[k])) return perr(std::string("non-finite value in '") + field_of[k] + "' at vertex " + std::to_string(v));
        }
        for (size_t r = 0; r < irest.size(); ++r)
            if (!std::isfinite((float)vals[irest[r]])) return perr("non-finite value in 'f_rest' at vertex " + std::to_string(v));
        // activated (gps-io lib.rs:84-96) + GpuGaussian::from_activated (gps.rs:41-49)
        gpsb_gaussian& g = splats[v];
        double op = 1.0 / (1.0 + exp(-(double)f[6]));
        g.pos_opacity[0] = f[0]; g.pos_opacity[1] = f[1]; g.pos_opacity[2] = f[2]; g.pos_opacity[3] = (float)op;
        g.log_scale[0] = f[7]; g.log_scale[1] = f[8]; g.log_scale[2] = f[9]; g.log_scale[3] = 0.0f;
        g.rot_wxyz[0] = f[10]; g.rot_wxyz[1] = f[11]; g.rot_wxyz[2] = f[12]; g.rot_wxyz[3] = f[13];
        for (int k = 0; k < 3; ++k) g.color[k] = (float)((double)f[3 + k] * kShC0 + 0.5);
        g.color[3] = 0.0f;
        if (sh_rest)
            for (size_t r = 0; r < irest.size(); ++r) sh_rest[v * 3 * per_ch + r] = (float)vals[irest[r]];
    }
    return GPSB_OK;
}

}  // extern "C"
