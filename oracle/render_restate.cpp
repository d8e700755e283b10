// CPU restatement of the flythrough renderer's ray march (TEST INFRASTRUCTURE ONLY).
//
// The checker of tg_viewer_render: given the window state the library reports
// (tg_viewer_state) and the same camera, it traces every pixel on the CPU and returns each
// pixel's first-ray hit and the frame. The traversal restates the reference renderer's
// algorithm (viz/fly.cu:124-182: Amanatides-Woo voxel stepping from the camera, whole 4 x 4
// column cells skipped while the ray stays above their highest block, water passed
// through with its entry distance kept, 6,000 steps at most); the shading restates the
// library's own model (shadow ray, face ambient occlusion, water tint and Fresnel
// reflection, haze, tone curve). Every operation of the traversal is a single IEEE float
// operation in the same order as the device code (built here with -ffp-contract=off), so
// hits agree exactly; the shading calls expf / powf / sqrtf of the host library, so colours
// agree to within a few units of the last u8 step.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

constexpr int kCell = 4;
constexpr int kMaxSteps = 6000;

struct World {
    const uint8_t* vox;
    const uint32_t* cell_top;
    const int32_t* slot;   // x, z pairs
    const int32_t* born;
    int W, WB, WC;
    int air, water, lava, bedrock;
    int min_y, height;
};

struct Cam {
    float px, py, pz, fx, fy, fz, rx, ry, rz, ux, uy, uz, tan_half, aspect, lx, ly, lz, fog;
};

struct Colours {
    float top[64][3], side[64][3];
    int cap[64];
};

int wrap(int a, int m) {
    const int r = a % m;
    return r < 0 ? r + m : r;
}
int floor_div(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

bool holds(const World& w, int x, int z) {
    const int cx = x >> 4, cz = z >> 4;
    const int k = wrap(cz, w.W) * w.W + wrap(cx, w.W);
    return w.slot[2 * k] == cx && w.slot[2 * k + 1] == cz;
}

int voxel(const World& w, int x, int y, int z) {
    const int yi = y - w.min_y;
    if (yi < 0) return w.bedrock;
    if (yi >= w.height || !holds(w, x, z)) return w.air;
    return w.vox[(static_cast<size_t>(yi) * w.WB + wrap(z, w.WB)) * w.WB + wrap(x, w.WB)];
}

int cell_top(const World& w, int x, int z) {
    if (!holds(w, x, z)) return w.min_y;
    return w.min_y + static_cast<int>(w.cell_top[wrap(floor_div(z, kCell), w.WC) * w.WC + wrap(floor_div(x, kCell), w.WC)]);
}

struct Hit {
    int id = 0, x = 0, y = 0, z = 0, nx = 0, ny = 0, nz = 0;
    float t = 0.0f, water_t = -1.0f;
};

bool trace(const World& w, float ox, float oy, float oz, float dx, float dy, float dz, float tmax, bool record_water, Hit& h) {
    const float ix = std::fabs(dx) > 1e-9f ? 1.0f / dx : 1e30f;
    const float iy = std::fabs(dy) > 1e-9f ? 1.0f / dy : 1e30f;
    const float iz = std::fabs(dz) > 1e-9f ? 1.0f / dz : 1e30f;
    const int sx = dx > 0.0f ? 1 : -1, sy = dy > 0.0f ? 1 : -1, sz = dz > 0.0f ? 1 : -1;
    const float ddx = std::fabs(ix), ddy = std::fabs(iy), ddz = std::fabs(iz);
    int vx = 0, vy = 0, vz = 0;
    float tx = 0, ty = 0, tz = 0;
    auto enter = [&](float t) {
        const float qx = ox + dx * t, qy = oy + dy * t, qz = oz + dz * t;
        vx = static_cast<int>(std::floor(qx));
        vy = static_cast<int>(std::floor(qy));
        vz = static_cast<int>(std::floor(qz));
        tx = (static_cast<float>(sx > 0 ? vx + 1 : vx) - ox) * ix;
        ty = (static_cast<float>(sy > 0 ? vy + 1 : vy) - oy) * iy;
        tz = (static_cast<float>(sz > 0 ? vz + 1 : vz) - oz) * iz;
    };
    float t = 0.0f;
    int nx = 0, ny = 0, nz = 0;
    enter(0.0f);
    h.water_t = -1.0f;
    const int top = w.min_y + w.height;
    for (int step = 0; step < kMaxSteps && t < tmax; ++step) {
        if (vy >= top) {
            if (dy >= 0.0f) return false;
        } else if (h.water_t < 0.0f) {
            const int ct = cell_top(w, vx, vz);
            if (vy >= ct) {
                const int cx = floor_div(vx, kCell), cz = floor_div(vz, kCell);
                const float ex = (static_cast<float>(sx > 0 ? (cx + 1) * kCell : cx * kCell) - ox) * ix;
                const float ez = (static_cast<float>(sz > 0 ? (cz + 1) * kCell : cz * kCell) - oz) * iz;
                const float te = std::fmin(ex, ez);
                if (oy + dy * te >= static_cast<float>(ct) && te > t) {
                    t = te + 1e-4f;
                    if (ex < ez) {
                        nx = -sx; ny = 0; nz = 0;
                    } else {
                        nx = 0; ny = 0; nz = -sz;
                    }
                    enter(t);
                    continue;
                }
            }
        }
        const int id = voxel(w, vx, vy, vz);
        if (id == w.water) {
            if (record_water && h.water_t < 0.0f) h.water_t = t;
        } else if (id != w.air) {
            h.id = id; h.x = vx; h.y = vy; h.z = vz; h.nx = nx; h.ny = ny; h.nz = nz; h.t = t;
            return true;
        }
        if (tx < ty && tx < tz) {
            vx += sx; t = tx; tx += ddx; nx = -sx; ny = 0; nz = 0;
        } else if (ty < tz) {
            vy += sy; t = ty; ty += ddy; nx = 0; ny = -sy; nz = 0;
        } else {
            vz += sz; t = tz; tz += ddz; nx = 0; ny = 0; nz = -sz;
        }
    }
    return false;
}

uint32_t hash4(int a, int b, int c, int d) {
    uint32_t h = static_cast<uint32_t>(a) * 0x9E3779B1u + static_cast<uint32_t>(b) * 0x85EBCA77u + static_cast<uint32_t>(c) * 0xC2B2AE3Du +
                 static_cast<uint32_t>(d) * 0x27D4EB2Fu;
    h ^= h >> 16; h *= 0x7FEB352Du; h ^= h >> 15; h *= 0x846CA68Bu; h ^= h >> 16;
    return h;
}
float fracf(float v) { return v - std::floor(v); }

void block_colour(const Colours& C, const Hit& h, float qx, float qy, float qz, float* out) {
    float u, v;
    int face;
    if (h.ny != 0) { u = fracf(qx); v = fracf(qz); face = h.ny > 0 ? 0 : 1; }
    else if (h.nx != 0) { u = fracf(qz); v = fracf(qy); face = 2; }
    else { u = fracf(qx); v = fracf(qy); face = 3; }
    const int tu = std::min(15, static_cast<int>(u * 16.0f)), tv = std::min(15, static_cast<int>(v * 16.0f));
    const float* c = C.top[h.id];
    if (C.cap[h.id] > 0 && h.ny <= 0) {
        const int rows = C.cap[h.id] - static_cast<int>(hash4(h.x, h.z, tu, 11) & 1u);
        if (h.ny < 0 || tv < 16 - rows) c = C.side[h.id];
    }
    const float texel = static_cast<float>(hash4(h.x * 16 + tu, h.y * 16 + tv, h.z, face) & 0xFFFFu) * (1.0f / 65535.0f);
    const float block = static_cast<float>(hash4(h.x, h.y, h.z, 7) & 0xFFFFu) * (1.0f / 65535.0f);
    const float k = 0.88f + 0.14f * texel + 0.05f * (block - 0.5f);
    for (int i = 0; i < 3; ++i) out[i] = c[i] * k;
}

float face_ao(const World& w, const Hit& h, float qx, float qy, float qz) {
    if (h.nx == 0 && h.ny == 0 && h.nz == 0) return 1.0f;
    const int fx = h.x + h.nx, fy = h.y + h.ny, fz = h.z + h.nz;
    int ux, uy, uz, vx, vy, vz;
    float fu, fv;
    if (h.nx != 0) { ux = 0; uy = 0; uz = 1; vx = 0; vy = 1; vz = 0; fu = fracf(qz); fv = fracf(qy); }
    else if (h.ny != 0) { ux = 1; uy = 0; uz = 0; vx = 0; vy = 0; vz = 1; fu = fracf(qx); fv = fracf(qz); }
    else { ux = 1; uy = 0; uz = 0; vx = 0; vy = 1; vz = 0; fu = fracf(qx); fv = fracf(qy); }
    auto solid = [&](int a, int b) {
        const int id = voxel(w, fx + a * ux + b * vx, fy + a * uy + b * vy, fz + a * uz + b * vz);
        return (id != w.air && id != w.water) ? 1 : 0;
    };
    const int e0 = solid(-1, 0), e1 = solid(1, 0), e2 = solid(0, -1), e3 = solid(0, 1);
    auto corner = [&](int a, int b, int ea, int eb) { return (ea && eb) ? 0.25f : 1.0f - 0.25f * static_cast<float>(ea + eb + solid(a, b)); };
    const float c00 = corner(-1, -1, e0, e2), c10 = corner(1, -1, e1, e2), c01 = corner(-1, 1, e0, e3), c11 = corner(1, 1, e1, e3);
    const float a0 = c00 + (c10 - c00) * fu, a1 = c01 + (c11 - c01) * fu;
    return a0 + (a1 - a0) * fv;
}

void sky(const Cam& cam, float dx, float dy, float dz, float* out) {
    const float up = std::fmax(dy, 0.0f);
    const float g = std::sqrt(up);
    out[0] = 0.62f + (0.16f - 0.62f) * g;
    out[1] = 0.74f + (0.33f - 0.74f) * g;
    out[2] = 0.92f + (0.70f - 0.92f) * g;
    if (dy < 0.0f) { out[0] = 0.58f; out[1] = 0.69f; out[2] = 0.86f; }
    const float s = std::fmax(dx * cam.lx + dy * cam.ly + dz * cam.lz, 0.0f);
    const float sun = std::pow(s, 1200.0f) * 10.0f + std::pow(s, 16.0f) * 0.15f;
    out[0] += 1.0f * sun;
    out[1] += 0.93f * sun;
    out[2] += 0.78f * sun;
}

uint8_t tone(float v) {
    const float x = std::fmax(v, 0.0f);
    const float m = x * (1.0f + x * 0.12f) / (1.0f + x);
    return static_cast<uint8_t>(std::fmin(255.0f, std::pow(std::fmin(m, 1.0f), 1.0f / 2.2f) * 255.0f + 0.5f));
}

void render_pixel(const World& w, const Cam& cam, const Colours& C, int width, int height, int frame, int px, int py, uint8_t* rgb, int32_t* hits) {
    float acc[3] = {0.0f, 0.0f, 0.0f};
    const float tmax = cam.fog * 1.05f;
    for (int s = 0; s < 4; ++s) {
        const float sxf = (static_cast<float>(px) + 0.25f + 0.5f * static_cast<float>(s & 1)) / static_cast<float>(width) * 2.0f - 1.0f;
        const float syf = 1.0f - (static_cast<float>(py) + 0.25f + 0.5f * static_cast<float>(s >> 1)) / static_cast<float>(height) * 2.0f;
        const float a = sxf * cam.tan_half * cam.aspect, b = syf * cam.tan_half;
        float dx = cam.fx + cam.rx * a + cam.ux * b;
        float dy = cam.fy + cam.ry * a + cam.uy * b;
        float dz = cam.fz + cam.rz * a + cam.uz * b;
        const float inv_len = 1.0f / std::sqrt(dx * dx + dy * dy + dz * dz);
        dx *= inv_len; dy *= inv_len; dz *= inv_len;
        Hit h;
        const bool hit = trace(w, cam.px, cam.py, cam.pz, dx, dy, dz, tmax, true, h);
        if (s == 0 && hits) {
            int32_t* o = hits + 4 * (static_cast<size_t>(py) * width + px);
            o[0] = hit ? h.id : -1; o[1] = hit ? h.x : 0; o[2] = hit ? h.y : 0; o[3] = hit ? h.z : 0;
        }
        float col[3];
        float dist = 1e30f;
        if (hit) {
            dist = h.t;
            const float qx = cam.px + dx * h.t, qy = cam.py + dy * h.t, qz = cam.pz + dz * h.t;
            float base[3];
            block_colour(C, h, qx, qy, qz, base);
            float ndl = std::fmax(static_cast<float>(h.nx) * cam.lx + static_cast<float>(h.ny) * cam.ly + static_cast<float>(h.nz) * cam.lz, 0.0f);
            if (ndl > 0.0f) {
                Hit sh;
                const float e = 0.002f;
                if (trace(w, qx + static_cast<float>(h.nx) * e, qy + static_cast<float>(h.ny) * e, qz + static_cast<float>(h.nz) * e, cam.lx, cam.ly, cam.lz, 256.0f,
                          false, sh))
                    ndl = 0.0f;
            }
            const float ao = face_ao(w, h, qx, qy, qz);
            const float face = h.ny > 0 ? 1.0f : (h.ny < 0 ? 0.5f : 0.75f);
            const float amb = face * (0.35f + 0.65f * ao);
            col[0] = base[0] * (1.40f * ndl + 0.32f * amb);
            col[1] = base[1] * (1.30f * ndl + 0.38f * amb);
            col[2] = base[2] * (1.12f * ndl + 0.50f * amb);
            if (h.id == w.lava) { col[0] = base[0] * 1.7f; col[1] = base[1] * 1.7f; col[2] = base[2] * 1.7f; }
            const int age = frame - w.born[wrap(h.z >> 4, w.W) * w.W + wrap(h.x >> 4, w.W)];
            if (age >= 0 && age < 8) col[1] += 0.08f * (1.0f - static_cast<float>(age) / 8.0f);
        } else {
            sky(cam, dx, dy, dz, col);
        }
        if (h.water_t >= 0.0f) {
            const float depth = (hit ? h.t : h.water_t + 48.0f) - h.water_t;
            const float tr = std::exp(-0.12f * depth);
            col[0] = col[0] * tr + 0.02f * (1.0f - tr);
            col[1] = col[1] * tr + 0.09f * (1.0f - tr);
            col[2] = col[2] * tr + 0.21f * (1.0f - tr);
            const float c = std::fabs(dy);
            const float F = 0.02f + 0.98f * std::pow(1.0f - c, 5.0f);
            float sk[3];
            sky(cam, dx, std::fabs(dy), dz, sk);
            for (int k = 0; k < 3; ++k) col[k] = col[k] * (1.0f - F) + sk[k] * F;
            dist = h.water_t;
        }
        if (dist < 1e29f && dist > 0.5f * cam.fog) {
            const float x = (dist - 0.5f * cam.fog) / (0.5f * cam.fog);
            const float f = 1.0f - std::exp(-2.0f * x * x);
            float sk[3];
            sky(cam, dx, std::fmax(dy, 0.02f), dz, sk);
            for (int k = 0; k < 3; ++k) col[k] = col[k] + (sk[k] - col[k]) * f;
        }
        for (int k = 0; k < 3; ++k) acc[k] += col[k];
    }
    uint8_t* o = rgb + (static_cast<size_t>(py) * width + px) * 3;
    o[0] = tone(acc[0] * 0.25f);
    o[1] = tone(acc[1] * 0.25f);
    o[2] = tone(acc[2] * 0.25f);
}

}  // namespace

extern "C" {

// cam: 18 floats {px, py, pz, fx, fy, fz, rx, ry, rz, ux, uy, uz, tan_half, aspect, lx, ly, lz, fog};
// ids: {W, air, water, lava, bedrock, min_y, height}; colours: 64 x 3 top, 64 x 3 side (floats),
// caps: 64 ints. rgb: width * height * 3; hits: width * height * 4 (may be null).
int rr_render(const uint8_t* vox, const uint32_t* cells, const int32_t* slots, const int32_t* born, const int32_t* ids, const float* cam_f, const float* top,
              const float* side, const int32_t* caps, int32_t width, int32_t height, int32_t frame, int32_t threads, uint8_t* rgb, int32_t* hits) {
    World w{vox, cells, slots, born, ids[0], ids[0] * 16, ids[0] * 4, ids[1], ids[2], ids[3], ids[4], ids[5], ids[6]};
    Cam cam;
    std::memcpy(&cam, cam_f, sizeof cam);
    Colours C;
    std::memcpy(C.top, top, sizeof C.top);
    std::memcpy(C.side, side, sizeof C.side);
    std::memcpy(C.cap, caps, sizeof C.cap);
    const int nt = threads > 0 ? threads : 1;
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; ++t)
        pool.emplace_back([&, t] {
            for (int py = t; py < height; py += nt)
                for (int px = 0; px < width; ++px) render_pixel(w, cam, C, width, height, frame, px, py, rgb, hits);
        });
    for (auto& th : pool) th.join();
    return 0;
}

}  // extern "C"
