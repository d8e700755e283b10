// Live flythrough renderer over generated terrain (device code).
//
// A toroidal voxel window of W x W chunks holds the generated blocks as u8 palette indices,
// [y][z][x] over the window's blocks; a chunk lands in slot (cz mod W, cx mod W), and a
// per-slot record of the chunk it holds makes every other chunk read as air. Per 4 x 4
// column cell the window keeps 1 + the highest non-air height index, for empty-space
// skipping. A frame is ray traced one thread per pixel with 2 x 2 supersampling: a
// voxel-by-voxel traversal (Amanatides-Woo) that skips whole column cells while the ray
// stays above their blocks, water seen through, then a shadow ray toward the sun, ambient
// occlusion from the eight neighbours in front of the hit face, water absorption and a
// Fresnel sky reflection, distance haze, and a filmic tone curve.
// Reference: the flythrough renderer viz/fly.cu (k_render :249-310, k_scatter :312-320,
// k_cells :322-334, its frame loop :486-560). The traversal follows the same algorithm;
// every float operation of the primary-ray traversal is IEEE-exact under this build's
// flags (no contraction, exact division and square root), so a CPU restatement reproduces
// each pixel's hit exactly.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tb {

constexpr int kViewCell = 4;          // empty-space cell side, in block columns
constexpr int kViewMaxSteps = 6000;   // traversal steps per ray
constexpr int kViewPalette = 64;

struct ViewWorld {
    uint8_t* vox;            // window voxels, [y][z][x]
    uint32_t* cell_top;      // per cell (z-major): 1 + highest non-air height index, 0 = empty
    const int2* slot;        // per window slot (cz mod W) * W + (cx mod W): the chunk it holds
    const int32_t* born;     // per slot: the frame its chunk was generated in
    int W, WB, WC;           // window side in chunks, blocks, cells
    int air, water, lava, bedrock;
};

struct ViewCam {
    float px, py, pz;        // eye
    float fx, fy, fz;        // forward (unit)
    float rx, ry, rz;        // right
    float ux, uy, uz;        // up
    float tan_half, aspect;  // vertical field of view, width / height
    float lx, ly, lz;        // unit direction to the sun
    float fog;               // haze distance (blocks); rays end at fog * 1.05
};

struct ViewColours {
    float top[kViewPalette][3];    // linear colour of top faces (of all faces when cap == 0)
    float side[kViewPalette][3];   // side and bottom colour of capped blocks (grass: dirt)
    int cap[kViewPalette];         // texel rows of the top colour at the top of side faces
};

__device__ __forceinline__ int vwrap(int a, int m) {
    const int r = a % m;
    return r < 0 ? r + m : r;
}
__device__ __forceinline__ int vfloor_div(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

__device__ __forceinline__ bool v_holds(const ViewWorld& w, int x, int z) {
    const int cx = x >> 4, cz = z >> 4;
    const int2 s = w.slot[vwrap(cz, w.W) * w.W + vwrap(cx, w.W)];
    return s.x == cx && s.y == cz;
}

__device__ __forceinline__ int v_voxel(const ViewWorld& w, int x, int y, int z) {
    const int yi = y - tbm::kMinY;
    if (yi < 0) return w.bedrock;
    if (yi >= tbm::kHeight || !v_holds(w, x, z)) return w.air;
    return w.vox[(static_cast<size_t>(yi) * w.WB + vwrap(z, w.WB)) * w.WB + vwrap(x, w.WB)];
}

// lowest absolute y at or above which the column cell of (x, z) holds only air
__device__ __forceinline__ int v_cell_top(const ViewWorld& w, int x, int z) {
    if (!v_holds(w, x, z)) return tbm::kMinY;
    return tbm::kMinY + static_cast<int>(w.cell_top[vwrap(vfloor_div(z, kViewCell), w.WC) * w.WC + vwrap(vfloor_div(x, kViewCell), w.WC)]);
}

struct ViewHit {
    int id, x, y, z, nx, ny, nz;
    float t;
    float water_t;   // distance where the ray entered water, -1 if it did not
};

// Traverses from o along unit d up to tmax; water is passed through (its entry distance
// recorded when record_water is set). Returns whether a non-air, non-water voxel was hit.
__device__ bool v_trace(const ViewWorld& w, float ox, float oy, float oz, float dx, float dy, float dz, float tmax, bool record_water, ViewHit& h) {
    const float ix = fabsf(dx) > 1e-9f ? 1.0f / dx : 1e30f;
    const float iy = fabsf(dy) > 1e-9f ? 1.0f / dy : 1e30f;
    const float iz = fabsf(dz) > 1e-9f ? 1.0f / dz : 1e30f;
    const int sx = dx > 0.0f ? 1 : -1, sy = dy > 0.0f ? 1 : -1, sz = dz > 0.0f ? 1 : -1;
    const float ddx = fabsf(ix), ddy = fabsf(iy), ddz = fabsf(iz);
    int vx, vy, vz;
    float tx, ty, tz;
    auto enter = [&](float t) {
        const float qx = ox + dx * t, qy = oy + dy * t, qz = oz + dz * t;
        vx = static_cast<int>(floorf(qx));
        vy = static_cast<int>(floorf(qy));
        vz = static_cast<int>(floorf(qz));
        tx = (static_cast<float>(sx > 0 ? vx + 1 : vx) - ox) * ix;
        ty = (static_cast<float>(sy > 0 ? vy + 1 : vy) - oy) * iy;
        tz = (static_cast<float>(sz > 0 ? vz + 1 : vz) - oz) * iz;
    };
    float t = 0.0f;
    int nx = 0, ny = 0, nz = 0;
    enter(0.0f);
    h.water_t = -1.0f;
    constexpr int top = tbm::kMinY + tbm::kHeight;
    for (int step = 0; step < kViewMaxSteps && t < tmax; ++step) {
        if (vy >= top) {
            if (dy >= 0.0f) return false;
        } else if (h.water_t < 0.0f) {
            const int ct = v_cell_top(w, vx, vz);
            if (vy >= ct) {
                // the ray may leave this column cell without coming down to its blocks
                const int cx = vfloor_div(vx, kViewCell), cz = vfloor_div(vz, kViewCell);
                const float ex = (static_cast<float>(sx > 0 ? (cx + 1) * kViewCell : cx * kViewCell) - ox) * ix;
                const float ez = (static_cast<float>(sz > 0 ? (cz + 1) * kViewCell : cz * kViewCell) - oz) * iz;
                const float te = fminf(ex, ez);
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
        const int id = v_voxel(w, vx, vy, vz);
        if (id == w.water) {
            if (record_water && h.water_t < 0.0f) h.water_t = t;
        } else if (id != w.air) {
            h.id = id;
            h.x = vx; h.y = vy; h.z = vz;
            h.nx = nx; h.ny = ny; h.nz = nz;
            h.t = t;
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

__device__ __forceinline__ uint32_t v_hash(int a, int b, int c, int d) {
    uint32_t h = static_cast<uint32_t>(a) * 0x9E3779B1u + static_cast<uint32_t>(b) * 0x85EBCA77u + static_cast<uint32_t>(c) * 0xC2B2AE3Du +
                 static_cast<uint32_t>(d) * 0x27D4EB2Fu;
    h ^= h >> 16;
    h *= 0x7FEB352Du;
    h ^= h >> 15;
    h *= 0x846CA68Bu;
    h ^= h >> 16;
    return h;
}

__device__ __forceinline__ float v_frac(float v) { return v - floorf(v); }

// surface colour of a hit: the block's face colour with per-texel and per-block variation
__device__ void v_block_colour(const ViewColours& C, const ViewHit& h, float qx, float qy, float qz, float* out) {
    float u, v;
    int face;
    if (h.ny != 0) {
        u = v_frac(qx); v = v_frac(qz); face = h.ny > 0 ? 0 : 1;
    } else if (h.nx != 0) {
        u = v_frac(qz); v = v_frac(qy); face = 2;
    } else {
        u = v_frac(qx); v = v_frac(qy); face = 3;
    }
    const int tu = min(15, static_cast<int>(u * 16.0f)), tv = min(15, static_cast<int>(v * 16.0f));
    const float* c = C.top[h.id];
    if (C.cap[h.id] > 0 && h.ny <= 0) {
        const int rows = C.cap[h.id] - static_cast<int>(v_hash(h.x, h.z, tu, 11) & 1u);
        if (h.ny < 0 || tv < 16 - rows) c = C.side[h.id];
    }
    const float texel = static_cast<float>(v_hash(h.x * 16 + tu, h.y * 16 + tv, h.z, face) & 0xFFFFu) * (1.0f / 65535.0f);
    const float block = static_cast<float>(v_hash(h.x, h.y, h.z, 7) & 0xFFFFu) * (1.0f / 65535.0f);
    const float k = 0.88f + 0.14f * texel + 0.05f * (block - 0.5f);
    out[0] = c[0] * k;
    out[1] = c[1] * k;
    out[2] = c[2] * k;
}

// light reaching the hit face from the sky: the fraction of its 4 edge and 4 corner
// neighbours (in front of the face) that are not solid, bilinear over the face
__device__ float v_face_ao(const ViewWorld& w, const ViewHit& h, float qx, float qy, float qz) {
    if (h.nx == 0 && h.ny == 0 && h.nz == 0) return 1.0f;
    const int fx = h.x + h.nx, fy = h.y + h.ny, fz = h.z + h.nz;
    int ux, uy, uz, vx, vy, vz;
    float fu, fv;
    if (h.nx != 0) {
        ux = 0; uy = 0; uz = 1; vx = 0; vy = 1; vz = 0; fu = v_frac(qz); fv = v_frac(qy);
    } else if (h.ny != 0) {
        ux = 1; uy = 0; uz = 0; vx = 0; vy = 0; vz = 1; fu = v_frac(qx); fv = v_frac(qz);
    } else {
        ux = 1; uy = 0; uz = 0; vx = 0; vy = 1; vz = 0; fu = v_frac(qx); fv = v_frac(qy);
    }
    auto solid = [&](int a, int b) {
        const int id = v_voxel(w, fx + a * ux + b * vx, fy + a * uy + b * vy, fz + a * uz + b * vz);
        return (id != w.air && id != w.water) ? 1 : 0;
    };
    const int e0 = solid(-1, 0), e1 = solid(1, 0), e2 = solid(0, -1), e3 = solid(0, 1);
    auto corner = [&](int a, int b, int ea, int eb) { return (ea && eb) ? 0.25f : 1.0f - 0.25f * static_cast<float>(ea + eb + solid(a, b)); };
    const float c00 = corner(-1, -1, e0, e2), c10 = corner(1, -1, e1, e2), c01 = corner(-1, 1, e0, e3), c11 = corner(1, 1, e1, e3);
    const float a0 = c00 + (c10 - c00) * fu, a1 = c01 + (c11 - c01) * fu;
    return a0 + (a1 - a0) * fv;
}

__device__ void v_sky(const ViewCam& cam, float dx, float dy, float dz, float* out) {
    const float up = fmaxf(dy, 0.0f);
    const float g = sqrtf(up);
    out[0] = 0.62f + (0.16f - 0.62f) * g;
    out[1] = 0.74f + (0.33f - 0.74f) * g;
    out[2] = 0.92f + (0.70f - 0.92f) * g;
    if (dy < 0.0f) {
        out[0] = 0.58f; out[1] = 0.69f; out[2] = 0.86f;
    }
    const float s = fmaxf(dx * cam.lx + dy * cam.ly + dz * cam.lz, 0.0f);
    const float sun = powf(s, 1200.0f) * 10.0f + powf(s, 16.0f) * 0.15f;
    out[0] += 1.0f * sun;
    out[1] += 0.93f * sun;
    out[2] += 0.78f * sun;
}

__device__ __forceinline__ uint8_t v_tone(float v) {
    const float x = fmaxf(v, 0.0f);
    const float m = x * (1.0f + x * 0.12f) / (1.0f + x);         // soft shoulder
    return static_cast<uint8_t>(fminf(255.0f, powf(fminf(m, 1.0f), 1.0f / 2.2f) * 255.0f + 0.5f));
}

// One frame. hits (may be null): per pixel the first subsample's primary hit, 4 ints
// {id (-1: none), x, y, z}.
__global__ void k_view_render(const ViewWorld w, const __grid_constant__ ViewCam cam, const ViewColours* __restrict__ colours, int width, int height,
                              int frame, uint8_t* rgb, int4* hits) {
    const int px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= width || py >= height) return;
    const ViewColours& C = *colours;
    float acc[3] = {0.0f, 0.0f, 0.0f};
    const float tmax = cam.fog * 1.05f;
    for (int s = 0; s < 4; ++s) {
        const float sxf = (static_cast<float>(px) + 0.25f + 0.5f * static_cast<float>(s & 1)) / static_cast<float>(width) * 2.0f - 1.0f;
        const float syf = 1.0f - (static_cast<float>(py) + 0.25f + 0.5f * static_cast<float>(s >> 1)) / static_cast<float>(height) * 2.0f;
        const float a = sxf * cam.tan_half * cam.aspect, b = syf * cam.tan_half;
        float dx = cam.fx + cam.rx * a + cam.ux * b;
        float dy = cam.fy + cam.ry * a + cam.uy * b;
        float dz = cam.fz + cam.rz * a + cam.uz * b;
        const float inv_len = 1.0f / sqrtf(dx * dx + dy * dy + dz * dz);
        dx *= inv_len;
        dy *= inv_len;
        dz *= inv_len;
        ViewHit h;
        const bool hit = v_trace(w, cam.px, cam.py, cam.pz, dx, dy, dz, tmax, true, h);
        if (s == 0 && hits) hits[static_cast<size_t>(py) * width + px] = hit ? make_int4(h.id, h.x, h.y, h.z) : make_int4(-1, 0, 0, 0);
        float col[3];
        float dist = 1e30f;
        if (hit) {
            dist = h.t;
            const float qx = cam.px + dx * h.t, qy = cam.py + dy * h.t, qz = cam.pz + dz * h.t;
            float base[3];
            v_block_colour(C, h, qx, qy, qz, base);
            float ndl = fmaxf(static_cast<float>(h.nx) * cam.lx + static_cast<float>(h.ny) * cam.ly + static_cast<float>(h.nz) * cam.lz, 0.0f);
            if (ndl > 0.0f) {
                ViewHit sh;
                const float e = 0.002f;
                if (v_trace(w, qx + static_cast<float>(h.nx) * e, qy + static_cast<float>(h.ny) * e, qz + static_cast<float>(h.nz) * e, cam.lx, cam.ly, cam.lz,
                            256.0f, false, sh))
                    ndl = 0.0f;
            }
            const float ao = v_face_ao(w, h, qx, qy, qz);
            const float face = h.ny > 0 ? 1.0f : (h.ny < 0 ? 0.5f : 0.75f);
            const float amb = face * (0.35f + 0.65f * ao);
            col[0] = base[0] * (1.40f * ndl + 0.32f * amb);
            col[1] = base[1] * (1.30f * ndl + 0.38f * amb);
            col[2] = base[2] * (1.12f * ndl + 0.50f * amb);
            if (h.id == w.lava) {
                col[0] = base[0] * 1.7f; col[1] = base[1] * 1.7f; col[2] = base[2] * 1.7f;
            }
            const int age = frame - w.born[vwrap(h.z >> 4, w.W) * w.W + vwrap(h.x >> 4, w.W)];
            if (age >= 0 && age < 8) {
                const float f = 1.0f - static_cast<float>(age) / 8.0f;
                col[1] += 0.08f * f;
            }
        } else {
            v_sky(cam, dx, dy, dz, col);
        }
        if (h.water_t >= 0.0f) {
            const float depth = (hit ? h.t : h.water_t + 48.0f) - h.water_t;
            const float tr = expf(-0.12f * depth);
            col[0] = col[0] * tr + 0.02f * (1.0f - tr);
            col[1] = col[1] * tr + 0.09f * (1.0f - tr);
            col[2] = col[2] * tr + 0.21f * (1.0f - tr);
            const float c = fabsf(dy);
            const float F = 0.02f + 0.98f * powf(1.0f - c, 5.0f);
            float sky[3];
            v_sky(cam, dx, fabsf(dy), dz, sky);
            for (int k = 0; k < 3; ++k) col[k] = col[k] * (1.0f - F) + sky[k] * F;
            dist = h.water_t;
        }
        if (dist < 1e29f && dist > 0.5f * cam.fog) {
            const float x = (dist - 0.5f * cam.fog) / (0.5f * cam.fog);
            const float f = 1.0f - expf(-2.0f * x * x);
            float sky[3];
            v_sky(cam, dx, fmaxf(dy, 0.02f), dz, sky);
            for (int k = 0; k < 3; ++k) col[k] = col[k] + (sky[k] - col[k]) * f;
        }
        for (int k = 0; k < 3; ++k) acc[k] += col[k];
    }
    uint8_t* o = rgb + (static_cast<size_t>(py) * width + px) * 3;
    o[0] = v_tone(acc[0] * 0.25f);
    o[1] = v_tone(acc[1] * 0.25f);
    o[2] = v_tone(acc[2] * 0.25f);
}

// New chunks into the window: chunk c of the batch's u16 states (< 256 by the palette
// size) as u8 voxels at its slot; 8 blocks per thread (one 16-byte load, one 8-byte store).
__global__ void k_view_scatter(ViewWorld w, const uint4* blocks, const int2* coords, int n) {
    constexpr int per8 = tbm::kHeight * 256 / 8;
    const long total = static_cast<long>(n) * per8;
    for (long t = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x; t < total; t += static_cast<long>(gridDim.x) * blockDim.x) {
        const int c = static_cast<int>(t / per8), e = static_cast<int>(t % per8) * 8;
        const int x = e & 15, z = (e >> 4) & 15, y = e >> 8;
        const uint4 v = blocks[static_cast<size_t>(c) * per8 + (e >> 3)];
        uint2 o;
        o.x = (v.x & 0xFFu) | ((v.x >> 8) & 0xFF00u) | ((v.y & 0xFFu) << 16) | ((v.y >> 16) << 24);
        o.y = (v.z & 0xFFu) | ((v.z >> 8) & 0xFF00u) | ((v.w & 0xFFu) << 16) | ((v.w >> 16) << 24);
        const int wx = vwrap(coords[c].x * 16 + x, w.WB), wz = vwrap(coords[c].y * 16 + z, w.WB);
        *reinterpret_cast<uint2*>(w.vox + (static_cast<size_t>(y) * w.WB + wz) * w.WB + wx) = o;
    }
}

// The 16 column cells of each new chunk set to empty, before k_view_cells.
__global__ void k_view_cells_clear(ViewWorld w, const int2* coords, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * 16) return;
    const int c = t >> 4, k = t & 15;
    const int bx = coords[c].x * 16 + (k & 3) * kViewCell, bz = coords[c].y * 16 + (k >> 2) * kViewCell;
    w.cell_top[vwrap(vfloor_div(bz, kViewCell), w.WC) * w.WC + vwrap(vfloor_div(bx, kViewCell), w.WC)] = 0;
}

// Per column of the new chunks: 1 + its highest non-air height index, folded into its cell
// by atomicMax.
__global__ void k_view_cells(ViewWorld w, const int2* coords, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * 256) return;
    const int c = t >> 8, x = t & 15, z = (t >> 4) & 15;
    const int bx = coords[c].x * 16 + x, bz = coords[c].y * 16 + z;
    const size_t col = static_cast<size_t>(vwrap(bz, w.WB)) * w.WB + vwrap(bx, w.WB);
    const size_t plane = static_cast<size_t>(w.WB) * w.WB;
    int top = 0;
    for (int y = tbm::kHeight - 1; y >= 0; --y)
        if (w.vox[y * plane + col] != w.air) {
            top = y + 1;
            break;
        }
    if (top) atomicMax(&w.cell_top[vwrap(vfloor_div(bz, kViewCell), w.WC) * w.WC + vwrap(vfloor_div(bx, kViewCell), w.WC)], static_cast<uint32_t>(top));
}

}  // namespace tb
