// host_geom.cpp -- see host_geom.h.
#include "host_geom.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

namespace hg
{

static const float kPi = 3.14159265358979323846f;

Camera camera_lookat(V3 pos, V3 target, float fov_deg)
{
    Camera c;
    c.pos = pos;
    c.fwd = normalize(target - pos);
    const V3 world_up = fabsf(c.fwd.y) < 0.99f ? V3(0.f, 1.f, 0.f) : V3(1.f, 0.f, 0.f);
    c.right = normalize(cross(c.fwd, world_up));
    c.up = cross(c.right, c.fwd);
    c.tan_half_fov_y = tanf(fov_deg * kPi / 180.f * 0.5f);
    return c;
}

Camera camera_quat(V3 pos, Q orient, float focal)
{
    Camera c;
    c.pos = pos;
    c.fwd = normalize(rotate(orient, V3(0.f, 0.f, -1.f)));
    c.right = normalize(rotate(orient, V3(1.f, 0.f, 0.f)));
    c.up = normalize(rotate(orient, V3(0.f, 1.f, 0.f)));
    c.tan_half_fov_y = 0.5f / focal;
    return c;
}

void store_camera(const Camera& c, rt_render_cfg* cfg)
{
    if (!cfg) { return; }
    const V3* src[4] = { &c.pos, &c.fwd, &c.right, &c.up };
    float* dst[4] = { cfg->cam_pos, cfg->cam_fwd, cfg->cam_right, cfg->cam_up };
    for (int i = 0; i < 4; i++) { dst[i][0] = src[i]->x; dst[i][1] = src[i]->y; dst[i][2] = src[i]->z; }
    cfg->tan_half_fov_y = c.tan_half_fov_y;
}

static rt_vertex mkv(float x, float y, float z, float nx, float ny, float nz)
{
    rt_vertex v;
    v.x = x; v.y = y; v.z = z; v.nx = nx; v.ny = ny; v.nz = nz;
    return v;
}
static rt_triangle mkt(uint32_t a, uint32_t b, uint32_t c)
{
    rt_triangle t;
    t.v[0] = a; t.v[1] = b; t.v[2] = c;
    return t;
}

// UV sphere of bvh_geo.cpp:22-112: north pole, rings-1 rings of `sectors` vertices, south
// pole; caps wound so the culling triangle test accepts hits from outside.
void add_sphere(std::vector<rt_vertex>& v, std::vector<rt_triangle>& t, V3 center, float radius, int rings, int sectors)
{
    const uint32_t off = (uint32_t)v.size();
    auto ring = [&](int r, int s) { return off + 1u + (uint32_t)((r - 1) * sectors + s); };
    v.push_back(mkv(center.x, center.y + radius, center.z, 0.f, 1.f, 0.f));
    for (int r = 1; r < rings; r++)
    {
        const float theta = kPi * (float)r / (float)rings;
        for (int s = 0; s < sectors; s++)
        {
            const float phi = 2.f * kPi * (float)s / (float)sectors;
            const float nx = sinf(theta) * cosf(phi);
            const float ny = cosf(theta);
            const float nz = sinf(theta) * sinf(phi);
            v.push_back(mkv(center.x + radius * nx, center.y + radius * ny, center.z + radius * nz, nx, ny, nz));
        }
    }
    const uint32_t south = (uint32_t)v.size();
    v.push_back(mkv(center.x, center.y - radius, center.z, 0.f, -1.f, 0.f));
    for (int s = 0; s < sectors; s++)
    {
        const int sn = (s + 1) % sectors;
        t.push_back(mkt(off, ring(1, sn), ring(1, s)));
    }
    for (int r = 1; r < rings - 1; r++)
    {
        for (int s = 0; s < sectors; s++)
        {
            const int sn = (s + 1) % sectors;
            const uint32_t a = ring(r, s), b = ring(r, sn), c = ring(r + 1, sn), d = ring(r + 1, s);
            t.push_back(mkt(a, b, c));
            t.push_back(mkt(a, c, d));
        }
    }
    for (int s = 0; s < sectors; s++)
    {
        const int sn = (s + 1) % sectors;
        t.push_back(mkt(south, ring(rings - 1, sn), ring(rings - 1, s)));
    }
}

// Oriented box of bvh_geo.cpp:114-192: 6 faces x 4 vertices (face normal as vertex normal),
// triangles (0,1,2) and (0,2,3) per face. Each face is given by its outward axis and sign and
// the signs of its four corners on the other two axes, walked so the faces point outward
// under the culling test.
void add_box(std::vector<rt_vertex>& v, std::vector<rt_triangle>& t, V3 center, V3 he, Q orient)
{
    // per face: normal (x,y,z) then 4 corners as sign triples (sx, sy, sz) multiplying he
    static const signed char kFaces[6][15] = {
        { 1, 0, 0, 1, 1, -1, 1, -1, -1, 1, -1, 1, 1, 1, 1 },
        { -1, 0, 0, -1, 1, 1, -1, -1, 1, -1, -1, -1, -1, 1, -1 },
        { 0, 1, 0, -1, 1, -1, -1, 1, 1, 1, 1, 1, 1, 1, -1 },
        { 0, -1, 0, -1, -1, 1, -1, -1, -1, 1, -1, -1, 1, -1, 1 },
        { 0, 0, 1, 1, 1, 1, 1, -1, 1, -1, -1, 1, -1, 1, 1 },
        { 0, 0, -1, -1, 1, -1, -1, -1, -1, 1, -1, -1, 1, 1, -1 },
    };
    auto sgn = [](signed char s, float h) { return s > 0 ? h : -h; };
    for (int f = 0; f < 6; f++)
    {
        const signed char* F = kFaces[f];
        const uint32_t off = (uint32_t)v.size();
        const V3 n = rotate(orient, V3((float)F[0], (float)F[1], (float)F[2]));
        for (int c = 0; c < 4; c++)
        {
            const signed char* s = F + 3 + 3 * c;
            const V3 corner(sgn(s[0], he.x), sgn(s[1], he.y), sgn(s[2], he.z));
            const V3 r = rotate(orient, corner);
            v.push_back(mkv(center.x + r.x, center.y + r.y, center.z + r.z, n.x, n.y, n.z));
        }
        t.push_back(mkt(off + 0, off + 1, off + 2));
        t.push_back(mkt(off + 0, off + 2, off + 3));
    }
}

std::string replace_extension(const std::string& path, const std::string& ext)
{
    const auto dot = path.rfind('.');
    return (dot != std::string::npos ? path.substr(0, dot) : path) + ext;
}

int read_scene(const std::string& path, std::vector<rt_vertex>& v, std::vector<rt_triangle>& t, std::string& err)
{
    std::ifstream file(path);
    if (!file.is_open())
    {
        std::fprintf(stderr, "Error : failed to open scene file %s on readScene()\n", path.c_str());
        err = "failed to open scene file " + path;
        return RT_E_IO;
    }
    std::string line;
    while (std::getline(file, line))
    {
        std::istringstream iss(line);
        std::string token;
        if (!(iss >> token)) { continue; }
        if (token == "sphere")
        {
            float cx, cy, cz, radius;
            if (!(iss >> cx >> cy >> cz >> radius))
            {
                std::fprintf(stderr, "Error : malformed sphere line on readScene()\n");
                continue;
            }
            int rings = 16, sectors = 32, r, s;
            if (iss >> r >> s) { rings = r; sectors = s; }
            if (rings < 2 || sectors < 3)
            {
                std::fprintf(stderr, "Error : sphere needs rings >= 2 and sectors >= 3 on readScene()\n");
                continue;
            }
            add_sphere(v, t, V3(cx, cy, cz), radius, rings, sectors);
            std::fprintf(stdout, "Info : Added Sphere\n");
            continue;
        }
        if (token == "box")
        {
            float cx, cy, cz, hx, hy, hz, qx, qy, qz, qw;
            std::string ot;
            if (!(iss >> cx >> cy >> cz >> hx >> hy >> hz >> ot >> qx >> qy >> qz >> qw))
            {
                std::fprintf(stderr, "Error : malformed box line on readScene()\n");
                continue;
            }
            if (ot != "q")
            {
                std::fprintf(stderr, "Warning : unknown orientation type '%s', defaulting to identity on readScene()\n", ot.c_str());
                qx = 0.f; qy = 0.f; qz = 0.f; qw = 1.f;
            }
            add_box(v, t, V3(cx, cy, cz), V3(hx, hy, hz), Q(qx, qy, qz, qw));
            std::fprintf(stdout, "Info : Added Box\n");
            continue;
        }
        if (token != "mesh") { continue; }
        std::string mesh_path, ot;
        float tx, ty, tz, scale, qx = 0.f, qy = 0.f, qz = 0.f, qw = 1.f;
        if (!(iss >> mesh_path >> tx >> ty >> tz >> scale >> ot)) { continue; }
        if (ot == "q") { iss >> qx >> qy >> qz >> qw; }
        else
        {
            std::fprintf(stderr, "Warning : unknown orientation type '%s', defaulting to identity on readScene()\n", ot.c_str());
        }
        std::fprintf(stdout, "Info : Found Mesh : %s\n", mesh_path.c_str());
        std::string e2;
        if (int e = load_ply(mesh_path, V3(tx, ty, tz), scale, Q(qx, qy, qz, qw), v, t, e2))
        {
            std::fprintf(stderr, "Error : failed to load mesh %s on readScene()\n", mesh_path.c_str());
            err = "failed to load mesh " + mesh_path + ": " + e2;
            return e;
        }
    }
    return RT_OK;
}

// ---- PLY ----------------------------------------------------------------------------------

namespace
{
struct PlyProp
{
    std::string name, type, count_type, item_type;
    bool is_list = false;
};
struct PlyElem
{
    std::string name;
    uint64_t count = 0;
    std::vector<PlyProp> props;
};

int type_size(const std::string& t)
{
    if (t == "char" || t == "uchar" || t == "int8" || t == "uint8") { return 1; }
    if (t == "short" || t == "ushort" || t == "int16" || t == "uint16") { return 2; }
    if (t == "int" || t == "uint" || t == "float" || t == "int32" || t == "uint32" || t == "float32") { return 4; }
    if (t == "double" || t == "float64") { return 8; }
    return 0;
}

double read_bin(const unsigned char* p, const std::string& t)
{
    if (t == "char" || t == "int8") { return (double)*(const int8_t*)p; }
    if (t == "uchar" || t == "uint8") { return (double)*p; }
    int16_t s16; uint16_t u16; int32_t s32; uint32_t u32; float f; double d;
    if (t == "short" || t == "int16") { std::memcpy(&s16, p, 2); return s16; }
    if (t == "ushort" || t == "uint16") { std::memcpy(&u16, p, 2); return u16; }
    if (t == "int" || t == "int32") { std::memcpy(&s32, p, 4); return s32; }
    if (t == "uint" || t == "uint32") { std::memcpy(&u32, p, 4); return u32; }
    if (t == "float" || t == "float32") { std::memcpy(&f, p, 4); return f; }
    std::memcpy(&d, p, 8);
    return d;
}

// 4x4 column-major float matrix with the reference's operation order (src/math/mat4.hpp)
struct M4 { float c[4][4]; };
M4 identity()
{
    M4 m;
    for (int i = 0; i < 4; i++) { for (int j = 0; j < 4; j++) { m.c[i][j] = i == j ? 1.f : 0.f; } }
    return m;
}
void mul_vec(const M4& m, const float v[4], float r[4])
{
    for (int k = 0; k < 4; k++) { r[k] = m.c[0][k] * v[0] + m.c[1][k] * v[1] + m.c[2][k] * v[2] + m.c[3][k] * v[3]; }
}
M4 mul(const M4& a, const M4& b)
{
    M4 r;
    for (int i = 0; i < 4; i++) { mul_vec(a, b.c[i], r.c[i]); }
    return r;
}
M4 quat_mat(Q q)
{
    const float xx = q.x * q.x, yy = q.y * q.y, zz = q.z * q.z;
    const float xy = q.x * q.y, xz = q.x * q.z, yz = q.y * q.z;
    const float wx = q.w * q.x, wy = q.w * q.y, wz = q.w * q.z;
    M4 m = identity();
    const float c0[4] = { 1.f - 2.f * (yy + zz), 2.f * (xy + wz), 2.f * (xz - wy), 0.f };
    const float c1[4] = { 2.f * (xy - wz), 1.f - 2.f * (xx + zz), 2.f * (yz + wx), 0.f };
    const float c2[4] = { 2.f * (xz + wy), 2.f * (yz - wx), 1.f - 2.f * (xx + yy), 0.f };
    for (int k = 0; k < 4; k++) { m.c[0][k] = c0[k]; m.c[1][k] = c1[k]; m.c[2][k] = c2[k]; }
    return m;
}
// inverse-transpose for normals, computed in double by Gauss-Jordan elimination
M4 inverse_transpose(const M4& m)
{
    double a[4][8];
    for (int r = 0; r < 4; r++)
    {
        for (int c = 0; c < 4; c++) { a[r][c] = m.c[c][r]; a[r][4 + c] = r == c ? 1.0 : 0.0; }
    }
    for (int col = 0; col < 4; col++)
    {
        int piv = col;
        for (int r = col + 1; r < 4; r++) { if (std::fabs(a[r][col]) > std::fabs(a[piv][col])) { piv = r; } }
        if (piv != col) { for (int c = 0; c < 8; c++) { std::swap(a[piv][c], a[col][c]); } }
        const double p = a[col][col];
        if (p == 0.0) { return identity(); }
        for (int c = 0; c < 8; c++) { a[col][c] /= p; }
        for (int r = 0; r < 4; r++)
        {
            if (r == col) { continue; }
            const double f = a[r][col];
            for (int c = 0; c < 8; c++) { a[r][c] -= f * a[col][c]; }
        }
    }
    M4 out;  // (inverse)^T in column-major: out.c[col][row] = inv[col][row]
    for (int r = 0; r < 4; r++) { for (int c = 0; c < 4; c++) { out.c[r][c] = (float)a[r][4 + c]; } }
    return out;
}
} // namespace

int load_ply(const std::string& path, V3 tr, float scale, Q orient, std::vector<rt_vertex>& v, std::vector<rt_triangle>& t,
             std::string& err)
{
    std::ifstream f(path, std::ios::binary);
    if (!f.is_open()) { err = "cannot open " + path; return RT_E_IO; }
    std::string line;
    std::getline(f, line);
    if (line.rfind("ply", 0) != 0) { err = "not a PLY file"; return RT_E_FORMAT; }
    bool binary = false;
    std::vector<PlyElem> elems;
    for (;;)
    {
        if (!std::getline(f, line)) { err = "truncated PLY header"; return RT_E_FORMAT; }
        if (!line.empty() && line.back() == '\r') { line.pop_back(); }
        std::istringstream ss(line);
        std::string kw;
        ss >> kw;
        if (kw == "format")
        {
            std::string fmt;
            ss >> fmt;
            if (fmt == "binary_little_endian") { binary = true; }
            else if (fmt != "ascii") { err = "unsupported PLY format " + fmt; return RT_E_FORMAT; }
        }
        else if (kw == "element")
        {
            PlyElem e;
            ss >> e.name >> e.count;
            elems.push_back(e);
        }
        else if (kw == "property" && !elems.empty())
        {
            PlyProp p;
            std::string ty;
            ss >> ty;
            if (ty == "list") { p.is_list = true; ss >> p.count_type >> p.item_type >> p.name; }
            else { p.type = ty; ss >> p.name; }
            elems.back().props.push_back(p);
        }
        else if (kw == "end_header") { break; }
    }
    const uint32_t voff = (uint32_t)v.size();
    std::vector<float> pos, nrm;
    std::vector<std::vector<uint32_t>> faces;
    bool has_n = false;
    for (const PlyElem& e : elems)
    {
        const bool is_v = e.name == "vertex", is_f = e.name == "face";
        int ix = -1, iy = -1, iz = -1, inx = -1, iny = -1, inz = -1, iidx = -1;
        for (size_t k = 0; k < e.props.size(); k++)
        {
            const std::string& n = e.props[k].name;
            if (n == "x") { ix = (int)k; } else if (n == "y") { iy = (int)k; } else if (n == "z") { iz = (int)k; }
            else if (n == "nx") { inx = (int)k; } else if (n == "ny") { iny = (int)k; } else if (n == "nz") { inz = (int)k; }
            else if (n == "vertex_indices" || n == "vertex_index") { iidx = (int)k; }
        }
        if (is_v) { has_n = inx >= 0 && iny >= 0 && inz >= 0; }
        for (uint64_t r = 0; r < e.count; r++)
        {
            std::vector<double> vals(e.props.size(), 0.0);
            std::vector<uint32_t> idx;
            for (size_t k = 0; k < e.props.size(); k++)
            {
                const PlyProp& p = e.props[k];
                if (p.is_list)
                {
                    double cnt;
                    std::vector<uint32_t> items;
                    if (binary)
                    {
                        unsigned char buf[8];
                        const int cs = type_size(p.count_type), is = type_size(p.item_type);
                        if (!cs || !is || !f.read((char*)buf, cs)) { err = "bad PLY list"; return RT_E_FORMAT; }
                        cnt = read_bin(buf, p.count_type);
                        for (int j = 0; j < (int)cnt; j++)
                        {
                            if (!f.read((char*)buf, is)) { err = "truncated PLY"; return RT_E_FORMAT; }
                            items.push_back((uint32_t)read_bin(buf, p.item_type));
                        }
                    }
                    else
                    {
                        if (!(f >> cnt)) { err = "truncated PLY"; return RT_E_FORMAT; }
                        for (int j = 0; j < (int)cnt; j++)
                        {
                            double x;
                            if (!(f >> x)) { err = "truncated PLY"; return RT_E_FORMAT; }
                            items.push_back((uint32_t)x);
                        }
                    }
                    if ((int)k == iidx) { idx = items; }
                }
                else
                {
                    if (binary)
                    {
                        unsigned char buf[8];
                        const int sz = type_size(p.type);
                        if (!sz || !f.read((char*)buf, sz)) { err = "truncated PLY"; return RT_E_FORMAT; }
                        vals[k] = read_bin(buf, p.type);
                    }
                    else if (!(f >> vals[k])) { err = "truncated PLY"; return RT_E_FORMAT; }
                }
            }
            if (is_v)
            {
                pos.push_back(ix >= 0 ? (float)vals[ix] : 0.f);
                pos.push_back(iy >= 0 ? (float)vals[iy] : 0.f);
                pos.push_back(iz >= 0 ? (float)vals[iz] : 0.f);
                if (has_n) { nrm.push_back((float)vals[inx]); nrm.push_back((float)vals[iny]); nrm.push_back((float)vals[inz]); }
            }
            else if (is_f) { faces.push_back(idx); }
        }
    }
    const uint32_t nv = (uint32_t)(pos.size() / 3);
    std::vector<rt_triangle> nt;
    for (const auto& fc : faces)
    {
        for (size_t j = 1; j + 1 < fc.size(); j++)
        {
            if (fc[0] >= nv || fc[j] >= nv || fc[j + 1] >= nv) { err = "PLY face index out of range"; return RT_E_FORMAT; }
            nt.push_back(mkt(fc[0], fc[j], fc[j + 1]));
        }
    }
    if (!has_n)
    {
        nrm.assign(pos.size(), 0.f);
        for (const rt_triangle& tri : nt)
        {
            const float* a = &pos[3 * tri.v[0]];
            const float* b = &pos[3 * tri.v[1]];
            const float* c = &pos[3 * tri.v[2]];
            const V3 n = cross(V3(b[0] - a[0], b[1] - a[1], b[2] - a[2]), V3(c[0] - a[0], c[1] - a[1], c[2] - a[2]));
            for (int k = 0; k < 3; k++)
            {
                nrm[3 * tri.v[k]] += n.x; nrm[3 * tri.v[k] + 1] += n.y; nrm[3 * tri.v[k] + 2] += n.z;
            }
        }
    }
    // transform = translate * scale * rotate (bvh_IO.cpp:221-224); normals by the inverse transpose
    M4 T = identity();
    for (int k = 0; k < 3; k++) { T.c[3][k] = (k == 0 ? tr.x : (k == 1 ? tr.y : tr.z)); }
    M4 S = identity();
    for (int k = 0; k < 3; k++) { S.c[k][k] = scale; }
    const M4 M = mul(mul(T, S), quat_mat(orient));
    const M4 NM = inverse_transpose(M);
    for (uint32_t i = 0; i < nv; i++)
    {
        const float p4[4] = { pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], 1.f };
        const float n4[4] = { nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2], 0.f };
        float tp[4], tn[4];
        mul_vec(M, p4, tp);
        mul_vec(NM, n4, tn);
        v.push_back(mkv(tp[0], tp[1], tp[2], tn[0], tn[1], tn[2]));
    }
    for (const rt_triangle& tri : nt) { t.push_back(mkt(voff + tri.v[0], voff + tri.v[1], voff + tri.v[2])); }
    return RT_OK;
}

// ---- Radiance RGBE images (Ward, "Real Pixels", Graphics Gems II, 1991) ----
// A pixel is three 8-bit mantissas sharing one exponent byte: for v = max(r, g, b) = m 2^e
// with m in [0.5, 1), the bytes are (r, g, b) * 256 m / v and e + 128. Scanlines of width
// 8..32767 are written run-length encoded per component ("new" RLE: 2, 2, width, then for each
// of the four planes runs of (128 + n, value) for n >= 4 repeats and literals (n, bytes...)).

static void to_rgbe(const float* c, unsigned char* o)
{
    const float v = std::max(c[0], std::max(c[1], c[2]));
    if (!(v >= 1e-32f)) { o[0] = o[1] = o[2] = o[3] = 0; return; }
    int e = 0;
    const float m = std::frexp(v, &e) * 256.0f / v;
    o[0] = (unsigned char)std::max(0.0f, c[0] * m);
    o[1] = (unsigned char)std::max(0.0f, c[1] * m);
    o[2] = (unsigned char)std::max(0.0f, c[2] * m);
    o[3] = (unsigned char)(e + 128);
}

static void from_rgbe(const unsigned char* in, float* c)
{
    if (in[3] == 0) { c[0] = c[1] = c[2] = 0.0f; return; }
    const float f = std::ldexp(1.0f, (int)in[3] - (128 + 8));
    c[0] = (float)in[0] * f; c[1] = (float)in[1] * f; c[2] = (float)in[2] * f;
}

static void rle_plane(const unsigned char* d, uint32_t n, std::vector<unsigned char>& out)
{
    uint32_t i = 0;
    while (i < n)
    {
        // find the next run of >= 4 equal bytes
        uint32_t run_at = i, run_len = 0;
        while (run_at < n)
        {
            run_len = 1;
            while (run_at + run_len < n && run_len < 127 && d[run_at + run_len] == d[run_at]) { run_len++; }
            if (run_len >= 4) { break; }
            run_at += run_len;
        }
        if (run_at >= n) { run_len = 0; run_at = n; }
        // literals before it, at most 128 per chunk
        while (i < run_at)
        {
            const uint32_t k = std::min<uint32_t>(128, run_at - i);
            out.push_back((unsigned char)k);
            out.insert(out.end(), d + i, d + i + k);
            i += k;
        }
        if (run_len >= 4)
        {
            out.push_back((unsigned char)(128 + run_len));
            out.push_back(d[run_at]);
            i = run_at + run_len;
        }
    }
}

int write_hdr(const std::string& path, const float* rgb, uint32_t w, uint32_t h, std::string& err)
{
    std::ofstream f(path, std::ios::binary);
    if (!f) { err = "cannot open " + path + " for writing"; return RT_E_IO; }
    std::ostringstream hdr;
    hdr << "#?RADIANCE\n# Written by librt_b200\nFORMAT=32-bit_rle_rgbe\nEXPOSURE=1.0\n\n-Y " << h << " +X " << w << "\n";
    const std::string hs = hdr.str();
    f.write(hs.data(), (std::streamsize)hs.size());
    std::vector<unsigned char> px((size_t)w * 4), plane(w), out;
    for (uint32_t y = 0; y < h; y++)
    {
        for (uint32_t x = 0; x < w; x++) { to_rgbe(rgb + 3 * ((size_t)y * w + x), &px[4 * (size_t)x]); }
        out.clear();
        if (w < 8 || w > 32767)
        {
            out.assign(px.begin(), px.end());
        }
        else
        {
            out.push_back(2); out.push_back(2); out.push_back((unsigned char)(w >> 8)); out.push_back((unsigned char)(w & 255));
            for (int c = 0; c < 4; c++)
            {
                for (uint32_t x = 0; x < w; x++) { plane[x] = px[4 * (size_t)x + c]; }
                rle_plane(plane.data(), w, out);
            }
        }
        f.write(reinterpret_cast<const char*>(out.data()), (std::streamsize)out.size());
    }
    if (!f) { err = "write failed: " + path; return RT_E_IO; }
    return RT_OK;
}

int read_hdr(const std::string& path, std::vector<float>& rgb, uint32_t& w, uint32_t& h, std::string& err)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) { err = "cannot open " + path; return RT_E_IO; }
    std::string line;
    if (!std::getline(f, line) || line.rfind("#?", 0) != 0) { err = path + ": not a Radiance file"; return RT_E_FORMAT; }
    bool fmt_ok = false;
    while (std::getline(f, line) && !line.empty())
    {
        if (line == "FORMAT=32-bit_rle_rgbe") { fmt_ok = true; }
    }
    if (!fmt_ok) { err = path + ": not 32-bit_rle_rgbe"; return RT_E_FORMAT; }
    if (!std::getline(f, line)) { err = path + ": no resolution line"; return RT_E_FORMAT; }
    long hh = 0, ww = 0;
    char ya[3] = { 0 }, xa[3] = { 0 };
    if (std::sscanf(line.c_str(), "%2s %ld %2s %ld", ya, &hh, xa, &ww) != 4 || std::string(ya) != "-Y" ||
        std::string(xa) != "+X" || hh <= 0 || ww <= 0 || hh > 65536 || ww > 65536)
    {
        err = path + ": unsupported resolution line '" + line + "'";
        return RT_E_FORMAT;
    }
    w = (uint32_t)ww; h = (uint32_t)hh;
    rgb.assign((size_t)w * h * 3, 0.0f);
    std::vector<unsigned char> px((size_t)w * 4);
    for (uint32_t y = 0; y < h; y++)
    {
        unsigned char head[4];
        if (!f.read(reinterpret_cast<char*>(head), 4)) { err = path + ": truncated"; return RT_E_FORMAT; }
        if (w >= 8 && w <= 32767 && head[0] == 2 && head[1] == 2 && ((uint32_t)head[2] << 8 | head[3]) == w)
        {
            for (int c = 0; c < 4; c++)
            {
                uint32_t x = 0;
                while (x < w)
                {
                    int cnt = f.get();
                    if (cnt == EOF) { err = path + ": truncated"; return RT_E_FORMAT; }
                    if (cnt > 128)
                    {
                        cnt -= 128;
                        const int v = f.get();
                        if (v == EOF || x + (uint32_t)cnt > w) { err = path + ": bad run"; return RT_E_FORMAT; }
                        for (int k = 0; k < cnt; k++) { px[4 * (size_t)(x++) + c] = (unsigned char)v; }
                    }
                    else
                    {
                        if (cnt == 0 || x + (uint32_t)cnt > w) { err = path + ": bad literal"; return RT_E_FORMAT; }
                        for (int k = 0; k < cnt; k++)
                        {
                            const int v = f.get();
                            if (v == EOF) { err = path + ": truncated"; return RT_E_FORMAT; }
                            px[4 * (size_t)(x++) + c] = (unsigned char)v;
                        }
                    }
                }
            }
        }
        else
        {
            std::memcpy(px.data(), head, 4);
            if (w > 1 && !f.read(reinterpret_cast<char*>(px.data() + 4), (std::streamsize)(4 * ((size_t)w - 1))))
            {
                err = path + ": truncated";
                return RT_E_FORMAT;
            }
        }
        for (uint32_t x = 0; x < w; x++) { from_rgbe(&px[4 * (size_t)x], &rgb[3 * ((size_t)y * w + x)]); }
    }
    return RT_OK;
}

SceneConfig parse_scene_config(const std::string& path)
{
    SceneConfig cfg;
    cfg.camera = camera_lookat(V3(0.f, 1.f, -5.f), V3(0.f, 0.f, 0.f), 60.f);
    std::ifstream f(path);
    if (!f.is_open()) { return cfg; }
    std::string line;
    while (std::getline(f, line))
    {
        std::istringstream iss(line);
        std::string token;
        if (!(iss >> token) || token[0] == '#') { continue; }
        if (token == "screen") { iss >> cfg.width >> cfg.height; }
        else if (token == "camera")
        {
            float px, py, pz;
            if (!(iss >> px >> py >> pz)) { continue; }
            std::string next;
            if (!(iss >> next)) { continue; }
            if (next == "lookat")
            {
                float tx, ty, tz, fov = 60.f;
                if (iss >> tx >> ty >> tz) { iss >> fov; }
                cfg.camera = camera_lookat(V3(px, py, pz), V3(tx, ty, tz), fov);
            }
            else
            {
                float focal = 0.f;
                try { focal = std::stof(next); } catch (...) { continue; }
                float qx = 0.f, qy = 0.f, qz = 0.f, qw = 1.f;
                std::string orient;
                if ((iss >> orient) && orient == "q") { iss >> qx >> qy >> qz >> qw; }
                cfg.camera = camera_quat(V3(px, py, pz), quat_normalize(Q(qx, qy, qz, qw)), focal);
            }
            cfg.has_camera = true;
        }
        else if (token == "ambient")
        {
            float r, g, b;
            if (iss >> r >> g >> b) { cfg.ambient[0] = r; cfg.ambient[1] = g; cfg.ambient[2] = b; }
        }
        else if (token == "ibl") { iss >> cfg.ibl_path; }
    }
    return cfg;
}

} // namespace hg
