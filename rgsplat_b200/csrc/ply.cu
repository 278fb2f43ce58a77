// ply.cu -- the model codecs of io::ply (src/io/ply.rs:35-303) for Gaussians
// that live on the device as float4 planes.
//
//   save_ply   (ply.rs:35-104): binary little-endian 3DGS layout, 62 f32 per
//              vertex (x y z, nx ny nz = 0, f_dc_0..2, f_rest_0..44
//              channel-major, opacity, scale_0..2, rot_0..3).
//   save_splat (ply.rs:253-285): 32-byte records: position, exp(log_scale),
//              RGBA bytes from the DC colour and sigmoid(opacity), quaternion
//              bytes of the normalised rotation.
//   load_ply   (ply.rs:116-193): any property order, binary LE / BE or ASCII;
//              each property decoded by its byte width alone (an int/uint is
//              read as f32 bits, char/short as unsigned) as the reference
//              does; unknown names are skipped; f_rest_i maps to channel i/15.
//
// The records are packed and unpacked on the device, straight from / into the
// planes: a CTA stages 128 PLY records in shared memory and writes them out
// contiguously, so only the file's bytes cross PCIe. Header text and ASCII
// bodies are handled on the host.
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "rgs_internal.cuh"
#include "rgs_math.cuh"

namespace rgs {

constexpr int PLY_FLOATS = 62;
constexpr int PLY_CTA = 128;
constexpr float SH_C0_F = 0.2820948f;  // ply.rs:24

__global__ void __launch_bounds__(PLY_CTA) k_pack_ply(const float4* __restrict__ params, int n, int cap, float* __restrict__ out) {
    __shared__ float s[PLY_CTA * PLY_FLOATS];
    const int tid = threadIdx.x;
    const int i0 = blockIdx.x * PLY_CTA, i = i0 + tid;
    if (i < n) {
        float r[59];
#pragma unroll
        for (int p = 0; p < NPL; ++p) {
            const float4 v = params[(size_t)p * cap + i];
            const float c[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int l = 0; l < 4; ++l) {
                // plane -> record index (record_to_plane inverted)
                const int f = p == 0 ? l : p == 1 ? 4 + l : p == 2 ? (l < 3 ? 8 + l : -1) : 11 + (p - 3) * 4 + l;
                if (f >= 0) r[f] = c[l];
            }
        }
        float* o = s + tid * PLY_FLOATS;
        o[0] = r[0]; o[1] = r[1]; o[2] = r[2];
        o[3] = 0.0f; o[4] = 0.0f; o[5] = 0.0f;
        o[6] = r[11]; o[7] = r[11 + 16]; o[8] = r[11 + 32];
#pragma unroll
        for (int ch = 0; ch < 3; ++ch)
#pragma unroll
            for (int k = 1; k < 16; ++k) o[9 + ch * 15 + (k - 1)] = r[11 + ch * 16 + k];
        o[54] = r[3];
        o[55] = r[8]; o[56] = r[9]; o[57] = r[10];
        o[58] = r[4]; o[59] = r[5]; o[60] = r[6]; o[61] = r[7];
    }
    __syncthreads();
    const int cnt = min(PLY_CTA, n - i0) * PLY_FLOATS;
    float* dst = out + (size_t)i0 * PLY_FLOATS;
    for (int k = tid; k < cnt; k += PLY_CTA) dst[k] = s[k];
}

// Rust `(x * 255.0).round() as u8` after a clamp that keeps NaN: round half
// away from zero, saturate, NaN -> 0.
__device__ __forceinline__ unsigned round_u8(float v) {
    const float r = roundf(v);
    if (!(r > 0.0f)) return 0u;
    if (r >= 255.0f) return 255u;
    return (unsigned)(int)r;
}

__global__ void __launch_bounds__(256) k_pack_splat(const float4* __restrict__ params, int n, int cap, uint4* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p0 = params[i], p1 = params[(size_t)cap + i], p2 = params[2 * (size_t)cap + i];
    const float dc_r = params[(size_t)3 * cap + i].x;    // sh[0]
    const float dc_g = params[(size_t)7 * cap + i].x;    // sh[16]
    const float dc_b = params[(size_t)11 * cap + i].x;   // sh[32]
    const unsigned cr = round_u8(rclamp(0.5f + dc_r * SH_C0_F, 0.0f, 1.0f) * 255.0f);
    const unsigned cg = round_u8(rclamp(0.5f + dc_g * SH_C0_F, 0.0f, 1.0f) * 255.0f);
    const unsigned cb = round_u8(rclamp(0.5f + dc_b * SH_C0_F, 0.0f, 1.0f) * 255.0f);
    const unsigned ca = round_u8(rclamp(sigmoid(p0.w), 0.0f, 1.0f) * 255.0f);
    const float q[4] = {p1.x, p1.y, p1.z, p1.w};
    float qn[4];
    qnormalize(q, qn);
    unsigned qb[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) qb[k] = round_u8(rclamp(qn[k] * 128.0f + 128.0f, 0.0f, 255.0f));
    out[2 * (size_t)i] = make_uint4(__float_as_uint(p0.x), __float_as_uint(p0.y), __float_as_uint(p0.z),
                                    __float_as_uint(exp_cr(p2.x)));
    out[2 * (size_t)i + 1] = make_uint4(__float_as_uint(exp_cr(p2.y)), __float_as_uint(exp_cr(p2.z)),
                                        cr | (cg << 8) | (cb << 16) | (ca << 24),
                                        qb[0] | (qb[1] << 8) | (qb[2] << 16) | (qb[3] << 24));
}

// One thread per vertex: Gaussian3D::new defaults, then every property in
// file order (a later duplicate wins), then the planes.
__global__ void __launch_bounds__(256) k_unpack_ply(const uint8_t* __restrict__ body, size_t stride, int n,
                                                    const PlyField* __restrict__ fields, int nfields, int big_endian,
                                                    float4* __restrict__ params, int cap) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float r[59];
#pragma unroll
    for (int k = 0; k < 59; ++k) r[k] = 0.0f;
    r[3] = -2.0f;
    r[4] = 1.0f;
    r[8] = r[9] = r[10] = -3.0f;
    const uint8_t* rec = body + (size_t)i * stride;
    for (int k = 0; k < nfields; ++k) {
        const PlyField f = fields[k];
        uint8_t x[8];
        for (int b = 0; b < f.width; ++b) x[b] = big_endian ? rec[f.offset + f.width - 1 - b] : rec[f.offset + b];
        float v;
        if (f.width == 4) {
            v = __uint_as_float((uint32_t)x[0] | ((uint32_t)x[1] << 8) | ((uint32_t)x[2] << 16) | ((uint32_t)x[3] << 24));
        } else if (f.width == 8) {
            unsigned long long u = 0;
            for (int b = 7; b >= 0; --b) u = (u << 8) | x[b];
            v = __double2float_rn(__longlong_as_double((long long)u));
        } else if (f.width == 1) {
            v = (float)x[0];
        } else {
            v = (float)((uint32_t)x[0] | ((uint32_t)x[1] << 8));
        }
        if (f.target >= 0) r[f.target] = v;
    }
#pragma unroll
    for (int p = 0; p < NPL; ++p) {
        float c[4];
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            const int f = p == 0 ? l : p == 1 ? 4 + l : p == 2 ? (l < 3 ? 8 + l : -1) : 11 + (p - 3) * 4 + l;
            c[l] = f >= 0 ? r[f] : 0.0f;
        }
        params[(size_t)p * cap + i] = make_float4(c[0], c[1], c[2], c[3]);
    }
}

void launch_pack_ply(const float4* params, int n, int cap, float* out, cudaStream_t st) {
    if (n <= 0) return;
    k_pack_ply<<<(n + PLY_CTA - 1) / PLY_CTA, PLY_CTA, 0, st>>>(params, n, cap, out);
}

void launch_pack_splat(const float4* params, int n, int cap, void* out, cudaStream_t st) {
    if (n <= 0) return;
    k_pack_splat<<<(n + 255) / 256, 256, 0, st>>>(params, n, cap, (uint4*)out);
}

void launch_unpack_ply(const uint8_t* body, size_t stride, int n, const PlyField* fields, int nfields, int big_endian,
                       float4* params, int cap, cudaStream_t st) {
    if (n <= 0) return;
    k_unpack_ply<<<(n + 255) / 256, 256, 0, st>>>(body, stride, n, fields, nfields, big_endian, params, cap);
}

// ---- host side: header text and ASCII bodies ------------------------------

std::string ply_header(size_t n) {
    std::string h = "ply\nformat binary_little_endian 1.0\nelement vertex " + std::to_string(n) + "\n";
    for (const char* p : {"x", "y", "z", "nx", "ny", "nz"}) h += std::string("property float ") + p + "\n";
    for (int i = 0; i < 3; ++i) h += "property float f_dc_" + std::to_string(i) + "\n";
    for (int i = 0; i < 45; ++i) h += "property float f_rest_" + std::to_string(i) + "\n";
    h += "property float opacity\n";
    for (int i = 0; i < 3; ++i) h += "property float scale_" + std::to_string(i) + "\n";
    for (int i = 0; i < 4; ++i) h += "property float rot_" + std::to_string(i) + "\n";
    h += "end_header\n";
    return h;
}

namespace {

std::vector<std::string> split_ws(const std::string& s) {
    std::vector<std::string> t;
    size_t i = 0;
    while (i < s.size()) {
        while (i < s.size() && isspace((unsigned char)s[i])) ++i;
        size_t j = i;
        while (j < s.size() && !isspace((unsigned char)s[j])) ++j;
        if (j > i) t.push_back(s.substr(i, j - i));
        i = j;
    }
    return t;
}

bool read_line(const std::vector<uint8_t>& d, size_t& pos, std::string& line) {
    line.clear();
    if (pos >= d.size()) return false;
    while (pos < d.size()) {
        const char c = (char)d[pos++];
        line.push_back(c);
        if (c == '\n') break;
    }
    return true;
}

// gaussian_from_props' name -> Gaussian3D record index (ply.rs:217-252); -1 = skipped
int target_of(const std::string& nm) {
    static const char* direct[] = {"x", "y", "z", "opacity", "rot_0", "rot_1", "rot_2", "rot_3", "scale_0", "scale_1", "scale_2"};
    static const int idx[] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10};
    for (int k = 0; k < 11; ++k)
        if (nm == direct[k]) return idx[k];
    if (nm == "f_dc_0") return 11;
    if (nm == "f_dc_1") return 11 + 16;
    if (nm == "f_dc_2") return 11 + 32;
    if (nm.compare(0, 7, "f_rest_") == 0 && nm.size() > 7) {
        size_t v = 0;
        for (size_t c = 7; c < nm.size(); ++c) {
            if (nm[c] < '0' || nm[c] > '9') return -1;
            v = v * 10 + (size_t)(nm[c] - '0');
            if (v > (1u << 30)) return -1;
        }
        const size_t ch = v / 15, k = v % 15;  // the reference assumes 15 per channel
        return ch < 3 ? (int)(11 + ch * 16 + 1 + k) : -1;
    }
    return -1;
}

}  // namespace

int parse_ply(const std::vector<uint8_t>& d, PlyLayout& L, std::string& err) {
    size_t pos = 0;
    std::string line;
    read_line(d, pos, line);
    {
        auto t = split_ws(line);
        if (!(t.size() == 1 && t[0] == "ply")) { err = "not a PLY file (missing magic)"; return -1; }
    }
    L = PlyLayout{};
    L.format = 2;
    for (;;) {
        if (!read_line(d, pos, line)) { err = "unexpected EOF in PLY header"; return -1; }
        auto t = split_ws(line);
        if (t.size() == 3 && t[0] == "format") {
            if (t[1] == "binary_little_endian") L.format = 0;
            else if (t[1] == "binary_big_endian") L.format = 1;
            else if (t[1] == "ascii") L.format = 2;
            else { err = "unsupported PLY format: " + t[1]; return -1; }
        } else if (t.size() == 3 && t[0] == "element" && t[1] == "vertex") {
            size_t v = 0;
            if (t[2].empty()) { err = "vertex count"; return -1; }
            for (char c : t[2]) {
                if (c < '0' || c > '9' || v > ((size_t)1 << 40)) { err = "vertex count"; return -1; }
                v = v * 10 + (size_t)(c - '0');
            }
            L.count = v;
        } else if (t.size() == 3 && t[0] == "property") {
            const std::string& ty = t[1];
            int w;
            if (ty == "float" || ty == "float32") w = 4;
            else if (ty == "double" || ty == "float64") w = 8;
            else if (ty == "uchar" || ty == "uint8" || ty == "char" || ty == "int8") w = 1;
            else if (ty == "short" || ty == "ushort" || ty == "int16" || ty == "uint16") w = 2;
            else if (ty == "int" || ty == "uint" || ty == "int32" || ty == "uint32") w = 4;
            else { err = "unsupported PLY property type: " + ty; return -1; }
            PlyField f;
            f.offset = (uint32_t)L.stride;
            f.width = (uint8_t)w;
            f.target = (int16_t)target_of(t[2]);
            L.fields.push_back(f);
            L.stride += (size_t)w;
        } else if (t.size() == 1 && t[0] == "end_header") {
            break;
        }
    }
    L.body = pos;
    if (L.format != 2 && L.count > 0 && L.stride > 0 && (d.size() - pos) / L.stride < L.count) {
        err = "PLY body shorter than its vertex count";
        return -1;
    }
    return 0;
}

void decode_ply_ascii(const std::vector<uint8_t>& d, const PlyLayout& L, float* out) {
    size_t pos = L.body;
    std::string line;
    for (size_t i = 0; i < L.count; ++i) {
        read_line(d, pos, line);
        float* r = out + i * NP;
        for (int k = 0; k < NP; ++k) r[k] = 0.0f;
        r[3] = -2.0f;
        r[4] = 1.0f;
        r[8] = r[9] = r[10] = -3.0f;
        auto toks = split_ws(line);
        for (size_t k = 0; k < L.fields.size(); ++k) {
            float v = 0.0f;
            if (k < toks.size()) {
                char* e = nullptr;
                const float x = strtof(toks[k].c_str(), &e);
                v = (e && *e == 0) ? x : 0.0f;
            }
            if (L.fields[k].target >= 0) r[L.fields[k].target] = v;
        }
    }
}

}  // namespace rgs
