// oracle/ply.hpp -- CPU restatement of the reference's model codecs (TEST
// INFRASTRUCTURE ONLY): io::ply::save_ply / load_ply / save_splat
// (src/io/ply.rs:35-303), as byte buffers so tests can compare files.
#pragma once
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "oracle.hpp"

namespace orc {
namespace ply {

constexpr float SH_C0 = 0.2820948f;  // ply.rs:24
constexpr int SH_PER_CHANNEL = 16;

inline void put_f32(std::vector<uint8_t>& b, float v) {
    uint8_t x[4];
    std::memcpy(x, &v, 4);  // little-endian host
    b.insert(b.end(), x, x + 4);
}

// ply.rs:35-104
inline std::vector<uint8_t> save_ply(const float* g, size_t n) {
    std::string h = "ply\nformat binary_little_endian 1.0\nelement vertex " + std::to_string(n) + "\n";
    for (const char* p : {"x", "y", "z", "nx", "ny", "nz"}) h += std::string("property float ") + p + "\n";
    for (int i = 0; i < 3; ++i) h += "property float f_dc_" + std::to_string(i) + "\n";
    for (int i = 0; i < (SH_PER_CHANNEL - 1) * 3; ++i) h += "property float f_rest_" + std::to_string(i) + "\n";
    h += "property float opacity\n";
    for (int i = 0; i < 3; ++i) h += "property float scale_" + std::to_string(i) + "\n";
    for (int i = 0; i < 4; ++i) h += "property float rot_" + std::to_string(i) + "\n";
    h += "end_header\n";
    std::vector<uint8_t> b(h.begin(), h.end());
    for (size_t i = 0; i < n; ++i) {
        const float* r = g + i * 59;  // position 0..2, opacity 3, rotation 4..7, log_scale 8..10, sh 11..58
        put_f32(b, r[0]); put_f32(b, r[1]); put_f32(b, r[2]);
        put_f32(b, 0.0f); put_f32(b, 0.0f); put_f32(b, 0.0f);
        put_f32(b, r[11]); put_f32(b, r[11 + 16]); put_f32(b, r[11 + 32]);
        for (int ch = 0; ch < 3; ++ch)
            for (int k = 1; k < SH_PER_CHANNEL; ++k) put_f32(b, r[11 + ch * 16 + k]);
        put_f32(b, r[3]);
        put_f32(b, r[8]); put_f32(b, r[9]); put_f32(b, r[10]);
        put_f32(b, r[4]); put_f32(b, r[5]); put_f32(b, r[6]); put_f32(b, r[7]);
    }
    return b;
}

// Rust `(x.clamp(0.0, 1.0) * 255.0).round() as u8` and the quaternion byte
// `((v * 128.0 + 128.0).clamp(0.0, 255.0)).round() as u8`: clamp keeps NaN,
// round is half away from zero, the cast saturates and maps NaN to 0.
inline uint8_t round_u8(float v) {
    float r = std::round(v);
    if (!(r > 0.0f)) return 0;
    if (r >= 255.0f) return 255;
    return (uint8_t)(int)r;
}

// ply.rs:253-285
inline std::vector<uint8_t> save_splat(const float* g, size_t n) {
    std::vector<uint8_t> b;
    b.reserve(n * 32);
    for (size_t i = 0; i < n; ++i) {
        const float* r = g + i * 59;
        put_f32(b, r[0]); put_f32(b, r[1]); put_f32(b, r[2]);
        for (int k = 0; k < 3; ++k) put_f32(b, t_exp(r[8 + k]));  // Gaussian3D::scale, mod.rs:72-78
        b.push_back(round_u8(rclamp(0.5f + r[11] * SH_C0, 0.0f, 1.0f) * 255.0f));
        b.push_back(round_u8(rclamp(0.5f + r[11 + 16] * SH_C0, 0.0f, 1.0f) * 255.0f));
        b.push_back(round_u8(rclamp(0.5f + r[11 + 32] * SH_C0, 0.0f, 1.0f) * 255.0f));
        b.push_back(round_u8(rclamp(sigmoid(r[3]), 0.0f, 1.0f) * 255.0f));
        float q[4];
        qnormalize(r + 4, q);  // quaternion.rs:10-17
        for (int k = 0; k < 4; ++k) b.push_back(round_u8(rclamp(q[k] * 128.0f + 128.0f, 0.0f, 255.0f)));
    }
    return b;
}

enum { PLY_OK = 0, PLY_EMAGIC = -10, PLY_EEOF = -11, PLY_EFORMAT = -12, PLY_ETYPE = -13, PLY_ECOUNT = -14, PLY_EBODY = -15 };

struct Prop {
    std::string name;
    int width;
};

// ply.rs:195-214 decode_scalar: only the byte width matters (an int/uint
// property is read as f32 bits, char / short as unsigned), as in the reference.
inline float decode_scalar(const uint8_t* p, int width, bool le) {
    uint8_t x[8];
    for (int i = 0; i < width; ++i) x[i] = le ? p[i] : p[width - 1 - i];
    if (width == 4) { float f; std::memcpy(&f, x, 4); return f; }
    if (width == 8) { double d; std::memcpy(&d, x, 8); return (float)d; }
    if (width == 1) return (float)x[0];
    if (width == 2) { uint16_t u; std::memcpy(&u, x, 2); return (float)u; }
    return 0.0f;
}

// ply.rs:217-252 gaussian_from_props (Gaussian3D::new defaults, mod.rs:52-62)
inline void gaussian_from_props(const std::vector<Prop>& props, const std::vector<float>& vals, float* r) {
    for (int k = 0; k < 59; ++k) r[k] = 0.0f;
    r[4] = 1.0f;
    r[8] = r[9] = r[10] = -3.0f;
    r[3] = -2.0f;
    for (size_t i = 0; i < props.size(); ++i) {
        const std::string& nm = props[i].name;
        const float v = i < vals.size() ? vals[i] : 0.0f;
        if (nm == "x") r[0] = v;
        else if (nm == "y") r[1] = v;
        else if (nm == "z") r[2] = v;
        else if (nm == "f_dc_0") r[11] = v;
        else if (nm == "f_dc_1") r[11 + 16] = v;
        else if (nm == "f_dc_2") r[11 + 32] = v;
        else if (nm == "opacity") r[3] = v;
        else if (nm == "scale_0") r[8] = v;
        else if (nm == "scale_1") r[9] = v;
        else if (nm == "scale_2") r[10] = v;
        else if (nm == "rot_0") r[4] = v;
        else if (nm == "rot_1") r[5] = v;
        else if (nm == "rot_2") r[6] = v;
        else if (nm == "rot_3") r[7] = v;
        else if (nm.compare(0, 7, "f_rest_") == 0 && nm.size() > 7) {
            // `str::parse::<usize>`: decimal digits only
            size_t idx = 0;
            bool ok = true;
            for (size_t c = 7; c < nm.size(); ++c) {
                if (nm[c] < '0' || nm[c] > '9') { ok = false; break; }
                idx = idx * 10 + (size_t)(nm[c] - '0');
            }
            if (ok) {
                const size_t ch = idx / 15, k = idx % 15;  // 15 f_rest per channel, as the reference assumes
                if (ch < 3) r[11 + ch * 16 + 1 + k] = v;
            }
        }
    }
}

inline std::vector<std::string> split_ws(const std::string& s) {
    std::vector<std::string> t;
    size_t i = 0;
    while (i < s.size()) {
        while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
        size_t j = i;
        while (j < s.size() && !std::isspace((unsigned char)s[j])) ++j;
        if (j > i) t.push_back(s.substr(i, j - i));
        i = j;
    }
    return t;
}

// ply.rs:116-193 load_ply
inline int load_ply(const uint8_t* data, size_t size, std::vector<float>& out) {
    size_t pos = 0;
    auto read_line = [&](std::string& line) -> bool {
        line.clear();
        if (pos >= size) return false;
        while (pos < size) {
            char c = (char)data[pos++];
            line.push_back(c);
            if (c == '\n') break;
        }
        return true;
    };
    std::string line;
    read_line(line);
    {
        auto t = split_ws(line);
        if (!(t.size() == 1 && t[0] == "ply")) return PLY_EMAGIC;
    }
    int fmt = 2;  // 0 binary LE, 1 binary BE, 2 ascii
    size_t count = 0;
    std::vector<Prop> props;
    for (;;) {
        if (!read_line(line)) return PLY_EEOF;
        auto t = split_ws(line);
        if (t.size() == 3 && t[0] == "format") {
            if (t[1] == "binary_little_endian") fmt = 0;
            else if (t[1] == "binary_big_endian") fmt = 1;
            else if (t[1] == "ascii") fmt = 2;
            else return PLY_EFORMAT;
        } else if (t.size() == 3 && t[0] == "element" && t[1] == "vertex") {
            const std::string& c = t[2];
            if (c.empty()) return PLY_ECOUNT;
            size_t v = 0;
            for (char ch : c) {
                if (ch < '0' || ch > '9') return PLY_ECOUNT;
                v = v * 10 + (size_t)(ch - '0');
            }
            count = v;
        } else if (t.size() == 3 && t[0] == "property") {
            const std::string& ty = t[1];
            int w;
            if (ty == "float" || ty == "float32") w = 4;
            else if (ty == "double" || ty == "float64") w = 8;
            else if (ty == "uchar" || ty == "uint8" || ty == "char" || ty == "int8") w = 1;
            else if (ty == "short" || ty == "ushort" || ty == "int16" || ty == "uint16") w = 2;
            else if (ty == "int" || ty == "uint" || ty == "int32" || ty == "uint32") w = 4;
            else return PLY_ETYPE;
            props.push_back({t[2], w});
        } else if (t.size() == 1 && t[0] == "end_header") {
            break;
        }
    }
    out.assign(count * 59, 0.0f);
    if (fmt == 2) {
        for (size_t i = 0; i < count; ++i) {
            read_line(line);
            std::vector<float> vals;
            for (auto& tok : split_ws(line)) {
                char* e = nullptr;
                float v = std::strtof(tok.c_str(), &e);
                vals.push_back((e && *e == 0) ? v : 0.0f);
            }
            gaussian_from_props(props, vals, out.data() + i * 59);
        }
    } else {
        size_t rw = 0;
        for (auto& p : props) rw += (size_t)p.width;
        std::vector<float> vals(props.size());
        for (size_t i = 0; i < count; ++i) {
            if (pos + rw > size) return PLY_EBODY;
            size_t off = 0;
            for (size_t k = 0; k < props.size(); ++k) {
                vals[k] = decode_scalar(data + pos + off, props[k].width, fmt == 0);
                off += (size_t)props[k].width;
            }
            pos += rw;
            gaussian_from_props(props, vals, out.data() + i * 59);
        }
    }
    return PLY_OK;
}

}  // namespace ply
}  // namespace orc
