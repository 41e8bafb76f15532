// io.cpp -- host-side scene and particle I/O in the reference's formats.
#include "io.hpp"

#include <algorithm>
#include <cctype>
#include <charconv>
#include <cmath>
#include <cstring>
#include <fstream>
#include <map>
#include <random>
#include <sstream>
#include <thread>

namespace fp::io {

namespace {
int label_code(char c) {
    switch (c) {
        case 'S': return FP_SOLID;
        case 'F': return FP_FLUID;
        case 'A': return FP_AIR;
        default: return -1;
    }
}
}  // namespace

bool read_labels3d(const std::string& path, int& W, int& H, int& D, std::vector<uint8_t>& out, std::string& err) {
    std::ifstream f(path);
    if (!f) { err = "cannot open label file: " + path; return false; }
    if (!(f >> W >> H >> D) || W <= 0 || H <= 0 || D <= 0) { err = "bad label header in " + path; return false; }
    const int64_t n = int64_t(W) * H * D;
    if (n > (int64_t(1) << 31)) { err = "label grid too large"; return false; }
    out.assign(size_t(n), FP_SOLID);
    for (int k = D - 1; k >= 0; --k)
        for (int j = H - 1; j >= 0; --j)
            for (int i = W - 1; i >= 0; --i) {
                char c;
                if (!(f >> c)) { err = "label file truncated: " + path; return false; }
                int l = label_code(c);
                if (l < 0) { err = std::string("unknown label character '") + c + "' in " + path; return false; }
                out[size_t(i) + size_t(j) * W + size_t(k) * W * H] = uint8_t(l);
            }
    return true;
}

bool read_labels2d(const std::string& path, int& W, int& H, std::vector<uint8_t>& out, std::string& err) {
    std::ifstream f(path);
    if (!f) { err = "cannot open label file: " + path; return false; }
    if (!(f >> W >> H) || W <= 0 || H <= 0) { err = "bad label header in " + path; return false; }
    out.assign(size_t(W) * H, FP_SOLID);
    for (int j = H - 1; j >= 0; --j)
        for (int i = 0; i < W; ++i) {
            char c;
            if (!(f >> c)) { err = "label file truncated: " + path; return false; }
            int l = label_code(c);
            if (l < 0) { err = std::string("unknown label character '") + c + "' in " + path; return false; }
            out[size_t(i) + size_t(j) * W] = uint8_t(l);
        }
    return true;
}

bool read_levelset2d(const std::string& path, char& kind, int& W, int& H, std::vector<float>& out, std::string& err) {
    std::ifstream f(path);
    if (!f) { err = "cannot open level-set file: " + path; return false; }
    std::string k;
    if (!(f >> k >> W >> H) || k.size() != 1 || W <= 0 || H <= 0) { err = "bad level-set header in " + path; return false; }
    kind = k[0];
    out.assign(size_t(W) * H, 0.0f);
    // rows in file order j = 0..h-1 of the generator; its row 0 is the top,
    // the order generate_combined_labels_simple writes and the 2D label reader reads
    for (int j = H - 1; j >= 0; --j)
        for (int i = 0; i < W; ++i) {
            float v;
            if (!(f >> v)) { err = "level-set file truncated: " + path; return false; }
            out[size_t(i) + size_t(j) * W] = v;
        }
    return true;
}

// ---------------------------------------------------------------- PLY
namespace {
int type_size(const std::string& t) {
    if (t == "char" || t == "uchar" || t == "int8" || t == "uint8") return 1;
    if (t == "short" || t == "ushort" || t == "int16" || t == "uint16") return 2;
    if (t == "int" || t == "uint" || t == "float" || t == "int32" || t == "uint32" || t == "float32") return 4;
    if (t == "double" || t == "float64") return 8;
    return 0;
}
double read_bin(const char* p, const std::string& t) {
    if (t == "float" || t == "float32") { float v; std::memcpy(&v, p, 4); return v; }
    if (t == "double" || t == "float64") { double v; std::memcpy(&v, p, 8); return v; }
    if (t == "int" || t == "int32") { int32_t v; std::memcpy(&v, p, 4); return v; }
    if (t == "uint" || t == "uint32") { uint32_t v; std::memcpy(&v, p, 4); return v; }
    if (t == "short" || t == "int16") { int16_t v; std::memcpy(&v, p, 2); return v; }
    if (t == "ushort" || t == "uint16") { uint16_t v; std::memcpy(&v, p, 2); return v; }
    if (t == "char" || t == "int8") { return double(int8_t(*p)); }
    return double(uint8_t(*p));
}
}  // namespace

bool read_ply(const std::string& path, std::vector<float>& pos, std::vector<float>& vel, bool& has_vel, std::string& err) {
    std::ifstream f(path, std::ios::binary);
    if (!f) { err = "cannot open PLY: " + path; return false; }
    std::string line;
    if (!std::getline(f, line) || line.rfind("ply", 0) != 0) { err = "not a PLY file: " + path; return false; }
    bool binary = false, in_vertex = false;
    int64_t nvert = -1;
    std::vector<std::pair<std::string, std::string>> props;  // (type, name) of the vertex element
    while (std::getline(f, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        std::istringstream ls(line);
        std::string kw;
        ls >> kw;
        if (kw == "format") {
            std::string fmt;
            ls >> fmt;
            if (fmt == "binary_little_endian") binary = true;
            else if (fmt != "ascii") { err = "unsupported PLY format " + fmt; return false; }
        } else if (kw == "element") {
            std::string name;
            int64_t cnt;
            ls >> name >> cnt;
            in_vertex = name == "vertex";
            if (in_vertex) nvert = cnt;
            else if (cnt > 0 && nvert >= 0) { /* trailing elements after vertices are ignored */ }
        } else if (kw == "property" && in_vertex) {
            std::string t, name;
            ls >> t;
            if (t == "list") { err = "list properties in the vertex element are not supported"; return false; }
            ls >> name;
            if (type_size(t) == 0) { err = "unknown PLY type " + t; return false; }
            props.emplace_back(t, name);
        } else if (kw == "end_header") {
            break;
        }
    }
    if (nvert < 0) { err = "PLY has no vertex element: " + path; return false; }
    int ix = -1, iy = -1, iz = -1, ivx = -1, ivy = -1, ivz = -1;
    for (size_t p = 0; p < props.size(); ++p) {
        const std::string& n = props[p].second;
        if (n == "x") ix = int(p); else if (n == "y") iy = int(p); else if (n == "z") iz = int(p);
        else if (n == "vx") ivx = int(p); else if (n == "vy") ivy = int(p); else if (n == "vz") ivz = int(p);
    }
    if (ix < 0 || iy < 0 || iz < 0) { err = "PLY vertices lack x y z"; return false; }
    has_vel = ivx >= 0 && ivy >= 0 && ivz >= 0;
    pos.assign(size_t(nvert) * 3, 0.0f);
    vel.assign(has_vel ? size_t(nvert) * 3 : 0, 0.0f);
    std::vector<double> rec(props.size());
    if (binary) {
        size_t rs = 0;
        std::vector<size_t> offs;
        for (auto& p : props) { offs.push_back(rs); rs += size_t(type_size(p.first)); }
        std::vector<char> buf(rs);
        for (int64_t v = 0; v < nvert; ++v) {
            if (!f.read(buf.data(), std::streamsize(rs))) { err = "PLY truncated at vertex " + std::to_string(v); return false; }
            for (size_t p = 0; p < props.size(); ++p) rec[p] = read_bin(buf.data() + offs[p], props[p].first);
            pos[3 * v] = float(rec[ix]); pos[3 * v + 1] = float(rec[iy]); pos[3 * v + 2] = float(rec[iz]);
            if (has_vel) { vel[3 * v] = float(rec[ivx]); vel[3 * v + 1] = float(rec[ivy]); vel[3 * v + 2] = float(rec[ivz]); }
        }
    } else {
        for (int64_t v = 0; v < nvert; ++v) {
            for (size_t p = 0; p < props.size(); ++p)
                if (!(f >> rec[p])) { err = "PLY truncated at vertex " + std::to_string(v); return false; }
            pos[3 * v] = float(rec[ix]); pos[3 * v + 1] = float(rec[iy]); pos[3 * v + 2] = float(rec[iz]);
            if (has_vel) { vel[3 * v] = float(rec[ivx]); vel[3 * v + 1] = float(rec[ivy]); vel[3 * v + 2] = float(rec[ivz]); }
        }
    }
    for (float x : pos) if (!std::isfinite(x)) { err = "PLY holds a non-finite coordinate"; return false; }
    return true;
}

namespace {
const char* kBinaryHeader =
    "\nproperty float x\nproperty float y\nproperty float z\nproperty float vx\nproperty float vy\n"
    "property float vz\nend_header\n";

// ASCII PLY / OFF of positions pos[stride * q + 0..2]: "x y z" per line as an
// ostream of floats prints them (save3dParticlesToPLY / save3dParticlesToOFF, utility.cu:91-127), %g
// with 6 significant digits, i.e. std::to_chars in general format with
// precision 6.  Chunks are formatted in parallel and written in order.
bool write_ascii(const std::string& path, const float* pos, int stride, int64_t n, int format, std::string& err) {
    std::ofstream f(path, std::ios::binary);
    if (!f) { err = "cannot write " + path; return false; }
    if (format == FP_OUT_OFF) {
        f << "OFF\n" << n << " 0 0\n";
    } else {
        f << "ply\nformat ascii 1.0\nelement vertex " << n << "\nproperty float x\nproperty float y\nproperty float z\nend_header\n";
    }
    const int64_t chunk = 1 << 18;
    const int64_t nchunks = (n + chunk - 1) / chunk;
    const int nthreads = int(std::max<int64_t>(1, std::min<int64_t>(nchunks, std::max(1u, std::thread::hardware_concurrency()))));
    std::vector<std::string> text(size_t(std::max<int64_t>(nchunks, 0)));
    auto format_chunk = [&](int64_t c) {
        std::string& out = text[size_t(c)];
        const int64_t b = c * chunk, e = std::min(n, b + chunk);
        out.resize(size_t(e - b) * 48);
        char* p = out.data();
        for (int64_t q = b; q < e; ++q)
            for (int a = 0; a < 3; ++a) {
                p = std::to_chars(p, p + 16, double(pos[stride * q + a]), std::chars_format::general, 6).ptr;
                *p++ = a < 2 ? ' ' : '\n';
            }
        out.resize(size_t(p - out.data()));
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; ++t)
        pool.emplace_back([&, t] {
            for (int64_t c = t; c < nchunks; c += nthreads) format_chunk(c);
        });
    for (auto& th : pool) th.join();
    for (const auto& s : text) f.write(s.data(), std::streamsize(s.size()));
    if (!f) { err = "write failed: " + path; return false; }
    return true;
}
}  // namespace

bool write_frame_records(const std::string& path, const float* rec, int64_t n, int format, std::string& err) {
    if (format == FP_OUT_NONE) return true;
    if (format != FP_OUT_PLY_BINARY) return write_ascii(path, rec, 6, n, format, err);
    std::ofstream f(path, std::ios::binary);
    if (!f) { err = "cannot write " + path; return false; }
    f << "ply\nformat binary_little_endian 1.0\nelement vertex " << n << kBinaryHeader;
    f.write(reinterpret_cast<const char*>(rec), std::streamsize(sizeof(float) * 6 * size_t(n)));
    if (!f) { err = "write failed: " + path; return false; }
    return true;
}

bool write_particles(const std::string& path, const float* pos, const float* vel, int64_t n, int format,
                     std::string& err) {
    if (format == FP_OUT_NONE) return true;
    if (format != FP_OUT_PLY_BINARY) return write_ascii(path, pos, 3, n, format, err);
    std::ofstream f(path, std::ios::binary);
    if (!f) { err = "cannot write " + path; return false; }
    f << "ply\nformat binary_little_endian 1.0\nelement vertex " << n << kBinaryHeader;
    std::vector<float> rec(size_t(6) * size_t(std::min<int64_t>(n, 1 << 16)));
    for (int64_t b = 0; b < n; b += (1 << 16)) {
        const int64_t m = std::min<int64_t>(n - b, 1 << 16);
        for (int64_t q = 0; q < m; ++q)
            for (int c = 0; c < 3; ++c) {
                rec[size_t(6 * q + c)] = pos[3 * (b + q) + c];
                rec[size_t(6 * q + 3 + c)] = vel ? vel[3 * (b + q) + c] : 0.0f;
            }
        f.write(reinterpret_cast<const char*>(rec.data()), std::streamsize(sizeof(float) * 6 * m));
    }
    if (!f) { err = "write failed: " + path; return false; }
    return true;
}

int64_t seed_particles(const uint8_t* labels, int W, int H, int D, float dx, int ppc, uint32_t seed,
                       std::vector<float>& pos) {
    pos.clear();
    std::mt19937 gen(seed);
    if (D > 1) {
        std::uniform_int_distribution<> sub(0, 7);
        std::uniform_real_distribution<> jit(-0.24f, 0.24f);
        const float o = 0.25f * dx;
        for (int k = 0; k < D; ++k)
            for (int j = 0; j < H; ++j)
                for (int i = 0; i < W; ++i) {
                    if (labels[size_t(i) + size_t(j) * W + size_t(k) * W * H] != FP_FLUID) continue;
                    const float cx = (i + 0.5f) * dx, cy = (j + 0.5f) * dx, cz = (k + 0.5f) * dx;
                    for (int q = 0; q < ppc; ++q) {
                        const int s = sub(gen);
                        const float jx = float(jit(gen) * dx), jy = float(jit(gen) * dx), jz = float(jit(gen) * dx);
                        float x = (cx + ((s & 1) ? o : -o)) + jx;
                        float y = (cy + ((s & 2) ? o : -o)) + jy;
                        float z = (cz + ((s & 4) ? o : -o)) + jz;
                        pos.push_back(std::clamp(x, i * dx, (i + 1) * dx));
                        pos.push_back(std::clamp(y, j * dx, (j + 1) * dx));
                        pos.push_back(std::clamp(z, k * dx, (k + 1) * dx));
                    }
                }
    } else {
        // 2D: quadrant centres (top-left, top-right, bottom-right, bottom-left),
        // clamped to the cell (FluidSolver2D.cu:114-158); z = 0.
        std::uniform_int_distribution<> sub(0, 3);
        std::uniform_real_distribution<> jit(-0.24f, 0.24f);
        for (int j = 0; j < H; ++j)
            for (int i = 0; i < W; ++i) {
                if (labels[size_t(i) + size_t(j) * W] != FP_FLUID) continue;
                const float cx = (i + 0.5f) * dx, cy = (j + 0.5f) * dx;
                const float sc[4][2] = {{cx - 0.25f * dx, cy + 0.25f * dx}, {cx + 0.25f * dx, cy + 0.25f * dx},
                                        {cx + 0.25f * dx, cy - 0.25f * dx}, {cx - 0.25f * dx, cy - 0.25f * dx}};
                for (int q = 0; q < ppc; ++q) {
                    const int s = sub(gen);
                    const float jx = float(jit(gen) * dx), jy = float(jit(gen) * dx);
                    float x = sc[s][0] + jx, y = sc[s][1] + jy;
                    pos.push_back(std::clamp(x, cx - 0.5f * dx, cx + 0.5f * dx));
                    pos.push_back(std::clamp(y, cy - 0.5f * dx, cy + 0.5f * dx));
                    pos.push_back(0.0f);
                }
            }
    }
    return int64_t(pos.size() / 3);
}

// ---------------------------------------------------------------- JSON
namespace {
struct JVal {
    enum { NUM, STR, BOOL, NUL, OTHER } kind = NUL;
    double num = 0;
    std::string str;
    bool b = false;
};
struct JParser {
    const std::string& s;
    size_t i = 0;
    std::string err;
    explicit JParser(const std::string& src) : s(src) {}
    void ws() { while (i < s.size() && std::isspace(static_cast<unsigned char>(s[i]))) ++i; }
    // Four hex digits at s[at]; false if they are missing or not hex.
    bool hex4(size_t at, uint32_t& v) const {
        if (at + 4 > s.size()) return false;
        v = 0;
        for (size_t k = at; k < at + 4; ++k) {
            const char c = s[k];
            const int d = c >= '0' && c <= '9' ? c - '0' : c >= 'a' && c <= 'f' ? c - 'a' + 10
                        : c >= 'A' && c <= 'F' ? c - 'A' + 10 : -1;
            if (d < 0) return false;
            v = v * 16 + uint32_t(d);
        }
        return true;
    }
    static void put_utf8(std::string& out, uint32_t cp) {
        if (cp < 0x80) {
            out += char(cp);
        } else if (cp < 0x800) {
            out += char(0xC0 | (cp >> 6));
            out += char(0x80 | (cp & 0x3F));
        } else if (cp < 0x10000) {
            out += char(0xE0 | (cp >> 12));
            out += char(0x80 | ((cp >> 6) & 0x3F));
            out += char(0x80 | (cp & 0x3F));
        } else {
            out += char(0xF0 | (cp >> 18));
            out += char(0x80 | ((cp >> 12) & 0x3F));
            out += char(0x80 | ((cp >> 6) & 0x3F));
            out += char(0x80 | (cp & 0x3F));
        }
    }
    // A JSON string with the escapes of RFC 8259 (as jsoncpp, which the
    // reference's driver uses, decodes them): \" \\ \/ \b \f \n \r \t and \uXXXX,
    // a surrogate pair giving one code point, written as UTF-8.  Any other
    // escape, or a lone surrogate, is an error.
    bool str(std::string& out) {
        if (i >= s.size() || s[i] != '"') return false;
        ++i;
        out.clear();
        while (i < s.size() && s[i] != '"') {
            if (s[i] != '\\') { out += s[i++]; continue; }
            if (i + 1 >= s.size()) return false;
            const char e = s[i + 1];
            i += 2;
            switch (e) {
                case '"': case '\\': case '/': out += e; break;
                case 'b': out += '\b'; break;
                case 'f': out += '\f'; break;
                case 'n': out += '\n'; break;
                case 'r': out += '\r'; break;
                case 't': out += '\t'; break;
                case 'u': {
                    uint32_t cp = 0;
                    if (!hex4(i, cp)) return false;
                    i += 4;
                    if (cp >= 0xD800 && cp < 0xDC00) {  // high surrogate: its low half must follow
                        uint32_t lo = 0;
                        if (i + 6 > s.size() || s[i] != '\\' || s[i + 1] != 'u' || !hex4(i + 2, lo) || lo < 0xDC00 ||
                            lo >= 0xE000)
                            return false;
                        i += 6;
                        cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                    } else if (cp >= 0xDC00 && cp < 0xE000) {
                        return false;
                    }
                    put_utf8(out, cp);
                    break;
                }
                default: return false;
            }
        }
        if (i >= s.size()) return false;
        ++i;
        return true;
    }
    bool skip_value(int depth = 0) {  // nested arrays/objects are skipped
        ws();
        if (i >= s.size() || depth > 64) return false;
        char c = s[i];
        if (c == '{' || c == '[') {
            char close = c == '{' ? '}' : ']';
            ++i;
            ws();
            if (i < s.size() && s[i] == close) { ++i; return true; }
            while (true) {
                if (c == '{') { std::string k; ws(); if (!str(k)) return false; ws(); if (i >= s.size() || s[i] != ':') return false; ++i; }
                if (!skip_value(depth + 1)) return false;
                ws();
                if (i < s.size() && s[i] == ',') { ++i; continue; }
                if (i < s.size() && s[i] == close) { ++i; return true; }
                return false;
            }
        }
        JVal v;
        return value(v);
    }
    bool value(JVal& v) {
        ws();
        if (i >= s.size()) return false;
        char c = s[i];
        if (c == '"') { v.kind = JVal::STR; return str(v.str); }
        if (s.compare(i, 4, "true") == 0) { v.kind = JVal::BOOL; v.b = true; i += 4; return true; }
        if (s.compare(i, 5, "false") == 0) { v.kind = JVal::BOOL; v.b = false; i += 5; return true; }
        if (s.compare(i, 4, "null") == 0) { v.kind = JVal::NUL; i += 4; return true; }
        if (c == '{' || c == '[') { v.kind = JVal::OTHER; return skip_value(); }
        size_t j = i;
        while (j < s.size() && (std::isdigit(static_cast<unsigned char>(s[j])) || s[j] == '-' || s[j] == '+' ||
                                s[j] == '.' || s[j] == 'e' || s[j] == 'E'))
            ++j;
        if (j == i) return false;
        v.kind = JVal::NUM;
        v.num = std::strtod(s.substr(i, j - i).c_str(), nullptr);
        i = j;
        return true;
    }
    bool object(std::map<std::string, JVal>& out) {
        ws();
        if (i >= s.size() || s[i] != '{') { err = "config is not a JSON object"; return false; }
        ++i;
        ws();
        if (i < s.size() && s[i] == '}') { ++i; return true; }
        while (true) {
            ws();
            std::string k;
            if (!str(k)) { err = "bad key"; return false; }
            ws();
            if (i >= s.size() || s[i] != ':') { err = "expected ':' after " + k; return false; }
            ++i;
            JVal v;
            if (!value(v)) { err = "bad value for " + k; return false; }
            out[k] = v;
            ws();
            if (i < s.size() && s[i] == ',') { ++i; continue; }
            if (i < s.size() && s[i] == '}') { ++i; return true; }
            err = "expected ',' or '}'";
            return false;
        }
    }
};
}  // namespace

bool load_config_json(const std::string& path, fp_config& cfg, std::string* label_path, int* frames, std::string& err) {
    std::ifstream f(path);
    if (!f) { err = "cannot open config: " + path; return false; }
    std::stringstream ss;
    ss << f.rdbuf();
    std::string text = ss.str();
    JParser p(text);
    std::map<std::string, JVal> m;
    if (!p.object(m)) { err = "config " + path + ": " + p.err; return false; }
    auto num = [&](const char* k, auto& dst) {
        auto it = m.find(k);
        if (it != m.end() && it->second.kind == JVal::NUM) dst = static_cast<std::remove_reference_t<decltype(dst)>>(it->second.num);
        else if (it != m.end() && it->second.kind == JVal::BOOL) dst = static_cast<std::remove_reference_t<decltype(dst)>>(it->second.b ? 1 : 0);
    };
    auto strv = [&](const char* k, std::string& dst) {
        auto it = m.find(k);
        if (it != m.end() && it->second.kind == JVal::STR) { dst = it->second.str; return true; }
        return false;
    };
    num("dt", cfg.dt);
    num("dx", cfg.dx);
    num("PIC_WEIGHT", cfg.pic_weight);
    num("iterPerFrame", cfg.iter_per_frame);
    std::string s;
    if (strv("outputFormat", s)) cfg.output_format = s == "PLY" ? FP_OUT_PLY : s == "PLY_BINARY" ? FP_OUT_PLY_BINARY
                                                   : s == "NONE" ? FP_OUT_NONE : FP_OUT_OFF;  // main.cpp:26-31
    if (strv("outputTemplate", s)) {
        std::snprintf(cfg.output_template, sizeof cfg.output_template, "%s", s.c_str());
    }
    if (label_path && strv("inputLabelData", s)) *label_path = s;
    if (strv("body_sdf", s)) std::snprintf(cfg.body_sdf, sizeof cfg.body_sdf, "%s", s.c_str());
    if (frames) num("frameAmount", *frames);
    num("activeBody", cfg.active_body);
    num("body_x", cfg.body_pos[0]);
    num("body_y", cfg.body_pos[1]);
    num("body_z", cfg.body_pos[2]);
    num("body_mass", cfg.body_mass);
    num("dim", cfg.dim);
    num("ppc", cfg.ppc);
    num("seed", cfg.seed);
    num("cfl", cfg.cfl);
    num("tol", cfg.tol);
    num("max_iters", cfg.max_iters);
    num("body_radius", cfg.body_radius);
    num("body_density", cfg.body_density);
    num("mg_sweeps", cfg.mg_sweeps);
    num("warm_start", cfg.warm_start);
    if (strv("solver", s)) {
        if (s == "pcg") cfg.solver = FP_SOLVER_PCG;
        else if (s == "pcg_mixed") cfg.solver = FP_SOLVER_PCG_MIXED;
        else if (s == "pcg_mg") cfg.solver = FP_SOLVER_PCG_MG;
        else if (s == "pcg_learned") cfg.solver = FP_SOLVER_PCG_LEARNED;
        else if (s == "pcg_learned_mixed") cfg.solver = FP_SOLVER_PCG_LEARNED_MIXED;
        else { err = "unknown solver " + s; return false; }
    }
    if (strv("collision", s)) {
        if (s == "labels") cfg.collision = FP_COLLISION_LABELS;
        else if (s == "sdf") cfg.collision = FP_COLLISION_SDF;
        else { err = "unknown collision " + s; return false; }
    }
    if (strv("advection", s)) {
        if (s == "rk3ref") cfg.advection = FP_ADVECT_RK3REF;
        else if (s == "rk2") cfg.advection = FP_ADVECT_RK2;
        else { err = "unknown advection " + s; return false; }
    }
    return true;
}

bool read_sdf(const std::string& path, int& w, int& h, int& d, float origin[3], float& cell, std::vector<float>& data,
              std::string& err) {
    std::ifstream f(path);
    if (!f) { err = "cannot open SDF file: " + path; return false; }
    if (!(f >> w >> h >> d) || w <= 0 || h <= 0 || d <= 0) { err = "bad SDF header"; return false; }
    if (!(f >> origin[0] >> origin[1] >> origin[2] >> cell) || !(cell > 0)) { err = "bad SDF origin/cell size"; return false; }
    data.assign(size_t(w) * h * d, 0.0f);
    for (size_t q = 0; q < data.size(); ++q)
        if (!(f >> data[q])) { err = "Unexpected end of SDF data"; return false; }  // utility.cuh:301
    return true;
}

}  // namespace fp::io
