// Headless screen-space fluid rendering for sm_100a: the reference app's OpenGL
// passes (src/renderapp.cpp:400-466) as CUDA kernels on device images.
//
//   pass                      reference shader             here
//   sprite depth + depth test shaders/depth.vert, .frag    k_splat<false>: one thread per
//                                                          particle, atomicMin on (depth, -z)
//   curvature-flow smoothing  shaders/smooth.frag (x60)    k_smooth, ping-pong images
//   additive thickness        shaders/thickness.frag       k_splat<true>: 64-bit fixed point
//   normals from depth        shaders/normal.frag          k_normals
//   room (background)         shaders/background.frag      k_room: one ray per pixel
//   fluid shading             shaders/shadingParticle.frag k_shade
//
// Images are width x height, row 0 at the bottom (the GL window convention);
// texture reads use the texel the reference's NEAREST / REPEAT sampling picks.
// Every expression keeps the shader's evaluation order (left to right, no fused
// multiply-add: the library is built with -fmad=false), so a CPU restatement in
// float32 reproduces the depth, smoothing, thickness, normal and room images bit
// for bit. Departures, all named:
//   * the depth test keeps the smallest (window depth, -z) pair, so equal depths
//     resolve the same way in any order (GL keeps the first fragment);
//   * thickness is summed in 64-bit fixed point (2^-24) so that the sum does not
//     depend on the order of the atomic adds (GL blends in float);
//   * sprites are at most 255 pixels wide and sprites whose centre lies outside
//     the near / far planes are dropped (GL clips points by their centre too);
//   * a pixel that no sprite covers takes the room colour: the reference shader
//     normalises a zero vector there;
//   * the room's colour is 0.95 everywhere (the reference gives two vertices of
//     the back wall a blue of 0.9).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdint>
#include <cstring>

#include "../../include/pbf.h"
#include "pbf_kernels.h"

namespace pbf {
namespace {

constexpr float kMaxSprite = 255.0f;
constexpr float kThickScale = 16777216.0f;  // 2^24

struct Cam {
    float V[16], P[16];
    float eye[3];
    float radius, pc, tan_half;
    float light[3], light_d[3];
    float roi;
    float room_light[3], room_light_d[3];
    float room[6];
    int w, h;
};

// rows of M (column-major) times (x, y, z, 1), left to right
__device__ __forceinline__ float row4(const float* M, int r, float x, float y, float z) {
    return ((M[r] * x + M[4 + r] * y) + M[8 + r] * z) + M[12 + r];
}
__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
    return (ax * bx + ay * by) + az * bz;
}

// Sprite depth (THICK false) or thickness (THICK true) of one particle per thread.
template <bool THICK>
__global__ void __launch_bounds__(256) k_splat(Cam c, const float* __restrict__ pos, int n, int stride,
                                               unsigned long long* __restrict__ depth,
                                               unsigned long long* __restrict__ thick) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* q = pos + (size_t)i * stride;
    const float px = q[0], py = q[1], pz = q[2];
    // depth.vert: viewPos = view * p; gl_Position = projection * viewPos
    const float vx = row4(c.V, 0, px, py, pz), vy = row4(c.V, 1, px, py, pz), vz = row4(c.V, 2, px, py, pz);
    if (!(vz < 0.0f)) return;
    const float cx = row4(c.P, 0, vx, vy, vz), cy = row4(c.P, 1, vx, vy, vz), cz = row4(c.P, 2, vx, vy, vz),
                cw = row4(c.P, 3, vx, vy, vz);
    if (!(cw > 0.0f)) return;
    const float ndz = cz / cw;
    if (!(ndz >= -1.0f && ndz <= 1.0f)) return;
    const float wx = (cx / cw + 1.0f) * 0.5f * (float)c.w;
    const float wy = (cy / cw + 1.0f) * 0.5f * (float)c.h;
    // gl_PointSize = -pointCoeff * radius / viewPos.z
    float size = -c.pc * c.radius / vz;
    size = fminf(fmaxf(size, 1.0f), kMaxSprite);
    const float half = 0.5f * size;
    if (!(wx + half >= 0.0f && wx - half <= (float)c.w && wy + half >= 0.0f && wy - half <= (float)c.h)) return;
    // pixels whose centres lie in [w - half, w + half)
    const int x0 = max((int)ceilf(wx - half - 0.5f), 0), x1 = min((int)ceilf(wx + half - 0.5f) - 1, c.w - 1);
    const int y0 = max((int)ceilf(wy - half - 0.5f), 0), y1 = min((int)ceilf(wy + half - 0.5f) - 1, c.h - 1);
    for (int yy = y0; yy <= y1; ++yy)
        for (int xx = x0; xx <= x1; ++xx) {
            // gl_PointCoord (origin at the upper left), then
            // vNormal.xy = vec2(2, -2) * gl_PointCoord + vec2(-1, 1)
            const float s = ((float)xx + 0.5f - wx) / size + 0.5f;
            const float t = 0.5f - ((float)yy + 0.5f - wy) / size;
            const float nx = 2.0f * s + -1.0f, ny = -2.0f * t + 1.0f;
            const float d2 = nx * nx + ny * ny;
            if (d2 > 1.0f) continue;
            const float nz = sqrtf(1.0f - d2);
            const size_t pix = (size_t)yy * c.w + xx;
            if (THICK) {
                // thickness = 2 * vNormal.z * radius, summed (GL_ONE, GL_ONE blending)
                const float th = 2.0f * nz * c.radius;
                atomicAdd(thick + pix, (unsigned long long)llrintf(th * kThickScale));
            } else {
                // surfacePos = viewPos.xyz + radius * vNormal; depth = -surfacePos.z
                const float sx = vx + c.radius * nx, sy = vy + c.radius * ny, sz = vz + c.radius * nz;
                const float qz = row4(c.P, 2, sx, sy, sz), qw = row4(c.P, 3, sx, sy, sz);
                float fd = 0.5f * (qz / qw) + 0.5f;  // gl_FragDepth
                fd = fminf(fmaxf(fd, 0.0f), 1.0f);
                const unsigned long long key =
                    ((unsigned long long)__float_as_uint(fd) << 32) | (unsigned long long)__float_as_uint(-sz);
                atomicMin(depth + pix, key);
            }
        }
}

__global__ void k_clear(unsigned long long* __restrict__ depth, unsigned long long* __restrict__ thick, size_t m) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    depth[i] = ~0ull;
    thick[i] = 0ull;
}

// depth texture (0 where no sprite: the reference clears it to 0) and thickness
__global__ void k_resolve(const unsigned long long* __restrict__ depth, const unsigned long long* __restrict__ thick,
                          float* __restrict__ z, float* __restrict__ zraw, float* __restrict__ th, size_t m) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const unsigned long long d = depth[i];
    const float v = d == ~0ull ? 0.0f : __uint_as_float((unsigned)(d & 0xffffffffull));
    z[i] = v;
    zraw[i] = v;
    th[i] = (float)(long long)thick[i] * (1.0f / kThickScale);
}

// texel (x, y) with GL_REPEAT wrapping
__device__ __forceinline__ float tex(const float* __restrict__ a, int x, int y, int w, int h) {
    x = x < 0 ? x + w : (x >= w ? x - w : x);
    y = y < 0 ? y + h : (y >= h ? y - h : y);
    return a[(size_t)y * w + x];
}

// smooth.frag: one explicit curvature-flow step of the depth image
__global__ void __launch_bounds__(256) k_smooth(const float* __restrict__ zin, float* __restrict__ zout, int w, int h,
                                                float Fx, float Fy) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= w) return;
    const float Cx = 2.0f / ((float)w * Fx), Cy = 2.0f / ((float)h * Fy);
    const float z = tex(zin, x, y, w, h);
    float out = 0.0f;
    if (z > 0.0f) {
        const float zpx = tex(zin, x + 1, y, w, h), zmx = tex(zin, x - 1, y, w, h);
        const float dzdx = (zpx == 0.0f || zmx == 0.0f) ? 0.0f : (zpx - zmx) * 0.5f;
        const float dz2dx2 = (zpx + zmx) - 2.0f * z;
        const float zpy = tex(zin, x, y + 1, w, h), zmy = tex(zin, x, y - 1, w, h);
        const float dzdy = (zpy == 0.0f || zmy == 0.0f) ? 0.0f : (zpy - zmy) * 0.5f;
        const float dz2dy2 = (zpy + zmy) - 2.0f * z;
        const float zpp = tex(zin, x + 1, y + 1, w, h), zpm = tex(zin, x + 1, y - 1, w, h);
        const float zmp = tex(zin, x - 1, y + 1, w, h), zmm = tex(zin, x - 1, y - 1, w, h);
        const float dz2dxdy = (((zpp + zmm) - zmp) - zpm) * 0.25f;
        const float nx = -Cy * dzdx, ny = Cx * dzdy, nz = (Cx * Cy) * z;
        const float D = dot3(nx, ny, nz, nx, ny, nz);
        const float Cx2 = Cx * Cx, Cy2 = Cy * Cy;
        const float dDdx = 2.0f * (((Cy2 * dzdx) * dz2dx2 + (Cx2 * dzdy) * dz2dxdy) + ((Cx2 * Cy2) * z) * dzdx);
        const float dDdy = 2.0f * (((Cy2 * dzdx) * dz2dxdy + (Cx2 * dzdy) * dz2dy2) + ((Cx2 * Cy2) * z) * dzdy);
        const float Ex = (0.5f * dzdx) * dDdx - dz2dx2 * D;
        const float Ey = (0.5f * dzdy) * dDdy - dz2dy2 * D;
        const float H = (0.5f * (Cy * Ex + Cx * Ey)) / (D * sqrtf(D));
        out = z - H * 0.01f;
        if (out < 0.0f) out = z;
    }
    zout[(size_t)y * w + x] = out;
}

// normal.frag
__global__ void __launch_bounds__(256) k_normals(const float* __restrict__ zin, float4* __restrict__ nrm, int w, int h,
                                                 float Fx, float Fy) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= w) return;
    const float Cx = 2.0f / ((float)w * Fx), Cy = 2.0f / ((float)h * Fy);
    const float z = tex(zin, x, y, w, h);
    float4 n = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (z > 0.0f) {
        const float zpx = tex(zin, x + 1, y, w, h), zmx = tex(zin, x - 1, y, w, h);
        const float dzdx = (zpx == 0.0f || zmx == 0.0f) ? 0.0f : (zpx - zmx) * 0.5f;
        const float zpy = tex(zin, x, y + 1, w, h), zmy = tex(zin, x, y - 1, w, h);
        const float dzdy = (zpy == 0.0f || zmy == 0.0f) ? 0.0f : (zpy - zmy) * 0.5f;
        const float nx = -Cy * dzdx, ny = Cx * dzdy, nz = (Cx * Cy) * z;
        const float len = sqrtf(dot3(nx, ny, nz, nx, ny, nz));
        n = make_float4(nx / len, ny / len, nz / len, 0.0f);
    }
    nrm[(size_t)y * w + x] = n;
}

__device__ __forceinline__ float quant8(float v) {  // an 8-bit normalised texel
    return rintf(fminf(fmaxf(v, 0.0f), 1.0f) * 255.0f) / 255.0f;
}

// The room of the reference app (left, right and back walls and the floor of a
// box, src/renderapp.cpp:58-85) lit by background.frag, one ray per pixel; the
// clear colour 0.75 where no wall is hit.
__global__ void __launch_bounds__(256) k_room(Cam c, float4* __restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= c.w) return;
    // view-space direction through the pixel centre, then to world space
    const float ux = (2.0f * ((float)x + 0.5f) / (float)c.w - 1.0f) / c.P[0];
    const float uy = (2.0f * ((float)y + 0.5f) / (float)c.h - 1.0f) / c.P[5];
    float d[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) d[a] = (c.V[4 * a] * ux + c.V[4 * a + 1] * uy) - c.V[4 * a + 2];
    const float* R = c.room;  // xmin ymin zmin xmax ymax zmax
    float best = 3.4e38f;
    float nrm[3] = {0.0f, 0.0f, 0.0f};
    // plane a = value, normal sign, and the two in-plane axes with their ranges
    auto hit = [&](int a, float v, float ns) {
        if (d[a] == 0.0f) return;
        const float t = (v - c.eye[a]) / d[a];
        if (!(t > 0.0f) || !(t < best)) return;
        const int b = (a + 1) % 3, e = (a + 2) % 3;
        const float pb = c.eye[b] + t * d[b], pe = c.eye[e] + t * d[e];
        if (pb < R[b] || pb > R[3 + b] || pe < R[e] || pe > R[3 + e]) return;
        best = t;
        nrm[0] = nrm[1] = nrm[2] = 0.0f;
        nrm[a] = ns;
    };
    hit(0, R[0], 1.0f);   // left wall, normal +x
    hit(0, R[3], -1.0f);  // right wall, normal -x
    hit(1, R[1], 1.0f);   // floor, normal +y
    hit(2, R[2], 1.0f);   // back wall, normal +z
    float4 col = make_float4(0.75f, 0.75f, 0.75f, 1.0f);
    if (best < 3.4e38f) {
        const float p0 = c.eye[0] + best * d[0], p1 = c.eye[1] + best * d[1], p2 = c.eye[2] + best * d[2];
        float lx = c.room_light[0] - p0, ly = c.room_light[1] - p1, lz = c.room_light[2] - p2;
        const float ll = sqrtf(dot3(lx, ly, lz, lx, ly, lz));
        lx = lx / ll; ly = ly / ll; lz = lz / ll;
        const float diff = fmaxf(dot3(lx, ly, lz, nrm[0], nrm[1], nrm[2]), 0.0f);
        col = make_float4(0.2f + (diff * c.room_light_d[0]) * 0.95f, 0.2f + (diff * c.room_light_d[1]) * 0.95f,
                          0.2f + (diff * c.room_light_d[2]) * 0.95f, 1.0f);
    }
    out[(size_t)y * c.w + x] = make_float4(quant8(col.x), quant8(col.y), quant8(col.z), 1.0f);
}

// shadingParticle.frag
__global__ void __launch_bounds__(256) k_shade(Cam c, const float* __restrict__ z_img,
                                               const float* __restrict__ th_img, const float4* __restrict__ n_img,
                                               const float4* __restrict__ room, float4* __restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= c.w) return;
    const size_t pix = (size_t)y * c.w + x;
    const float z = z_img[pix];
    if (!(z > 0.0f)) {
        out[pix] = room[pix];
        return;
    }
    const float u = ((float)x + 0.5f) / (float)c.w, v = ((float)y + 0.5f) / (float)c.h;
    const float4 n = n_img[pix];
    const float sx = (2.0f * u - 1.0f) * c.tan_half * z, sy = (2.0f * v - 1.0f) * c.tan_half * z, sz = -z;
    float vx = -sx, vy = -sy, vz = -sz;
    const float vl = sqrtf(dot3(vx, vy, vz, vx, vy, vz));
    vx = vx / vl; vy = vy / vl; vz = vz / vl;
    const float lpx = row4(c.V, 0, c.light[0], c.light[1], c.light[2]);
    const float lpy = row4(c.V, 1, c.light[0], c.light[1], c.light[2]);
    const float lpz = row4(c.V, 2, c.light[0], c.light[1], c.light[2]);
    float lx = lpx - sx, ly = lpy - sy, lz = lpz - sz;
    const float ll = sqrtf(dot3(lx, ly, lz, lx, ly, lz));
    lx = lx / ll; ly = ly / ll; lz = lz / ll;
    const float cf[3] = {0.1f, 0.4f, 0.8f};
    const float thickness = 0.08f * th_img[pix];
    const float beta = 0.01f * thickness;
    // backgroundTex at texCoord + beta * n.xy (NEAREST, REPEAT)
    int bx = (int)floorf((u + beta * n.x) * (float)c.w) % c.w, by = (int)floorf((v + beta * n.y) * (float)c.h) % c.h;
    bx = bx < 0 ? bx + c.w : bx;
    by = by < 0 ? by + c.h : by;
    const float4 S = room[(size_t)by * c.w + bx];
    const float e = expf(-thickness);
    const float a[3] = {cf[0] * (1.0f - e) + S.x * e, cf[1] * (1.0f - e) + S.y * e, cf[2] * (1.0f - e) + S.z * e};
    const float cosv = fminf(fmaxf(dot3(n.x, n.y, n.z, vx, vy, vz), 0.0f), 1.0f);
    const float f = (1.0f - c.roi) / (1.0f + c.roi);
    const float FF = f * f;
    const float F = FF * (1.0f - FF) * powf(1.0f - cosv, 5.0f);
    const float diff = fmaxf(dot3(lx, ly, lz, n.x, n.y, n.z), 0.0f);
    // reflect(-l, n) = -l - 2 dot(n, -l) n
    const float dn = dot3(n.x, n.y, n.z, -lx, -ly, -lz);
    const float rx = -lx - 2.0f * dn * n.x, ry = -ly - 2.0f * dn * n.y, rz = -lz - 2.0f * dn * n.z;
    const float spec = powf(fmaxf(dot3(vx, vy, vz, rx, ry, rz), 0.0f), 32.0f);
    float o[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) o[k] = (a[k] * (1.0f - F) + ((diff * c.light_d[k]) * cf[k]) * F) + spec;
    out[pix] = make_float4(o[0], o[1], o[2], 1.0f);
}

Cam make_cam(const pbf_camera& in, int w, int h) {
    Cam c{};
    std::memcpy(c.V, in.view, sizeof c.V);
    std::memcpy(c.P, in.proj, sizeof c.P);
    std::memcpy(c.eye, in.cam_pos, sizeof c.eye);
    c.radius = in.radius;
    c.pc = in.point_coeff;
    c.tan_half = in.tan_half_fov;
    std::memcpy(c.light, in.light_pos, sizeof c.light);
    std::memcpy(c.light_d, in.light_diffuse, sizeof c.light_d);
    c.roi = in.roi;
    std::memcpy(c.room_light, in.room_light_pos, sizeof c.room_light);
    std::memcpy(c.room_light_d, in.room_light_diffuse, sizeof c.room_light_d);
    std::memcpy(c.room, in.room, sizeof c.room);
    c.w = w;
    c.h = h;
    return c;
}

}  // namespace
}  // namespace pbf

struct pbf_render {
    int w = 0, h = 0;
    unsigned long long *depth = nullptr, *thick64 = nullptr;
    float *zraw = nullptr, *z0 = nullptr, *z1 = nullptr, *thick = nullptr;
    float4 *normal = nullptr, *room = nullptr, *color = nullptr;
    const float* zfinal = nullptr;  // the smoothed depth of the last frame
    cudaStream_t last = nullptr;
};

namespace {

int rfail(int code, const char* msg) { return pbf::set_last_error(code, msg); }

void rfree(pbf_render* r) {
    void* ptrs[] = {r->depth, r->thick64, r->zraw, r->z0, r->z1, r->thick, r->normal, r->room, r->color};
    for (void* p : ptrs)
        if (p) cudaFree(p);
}

bool finite_cam(const pbf_camera* c) {
    const float* f = reinterpret_cast<const float*>(c);
    const size_t nf = offsetof(pbf_camera, smooth_iterations) / sizeof(float);
    for (size_t i = 0; i < nf; ++i)
        if (!(f[i] == f[i]) || f[i] > 3.4e38f || f[i] < -3.4e38f) return false;
    return true;
}

int render_points(pbf_render* r, const float* pos, int n, int stride, const pbf_camera* cam, cudaStream_t st) {
    using namespace pbf;
    if (!r || !cam) return rfail(PBF_ERR_INVALID, "null argument");
    if (n < 0 || (n > 0 && !pos)) return rfail(PBF_ERR_INVALID, "bad particle array");
    if (stride < 3) return rfail(PBF_ERR_INVALID, "stride must be >= 3 floats");
    if (!finite_cam(cam)) return rfail(PBF_ERR_INVALID, "non-finite camera");
    if (cam->smooth_iterations < 0 || cam->smooth_iterations > 1000)
        return rfail(PBF_ERR_INVALID, "smooth_iterations must lie in [0, 1000]");
    if (!(cam->radius > 0.0f) || !(cam->point_coeff > 0.0f)) return rfail(PBF_ERR_INVALID, "radius and point_coeff must be positive");
    const Cam c = make_cam(*cam, r->w, r->h);
    const size_t m = (size_t)r->w * r->h;
    const int b1 = (int)((m + 255) / 256);
    k_clear<<<b1, 256, 0, st>>>(r->depth, r->thick64, m);
    if (n > 0) {
        k_splat<false><<<(n + 255) / 256, 256, 0, st>>>(c, pos, n, stride, r->depth, r->thick64);
        k_splat<true><<<(n + 255) / 256, 256, 0, st>>>(c, pos, n, stride, r->depth, r->thick64);
    }
    k_resolve<<<b1, 256, 0, st>>>(r->depth, r->thick64, r->z0, r->zraw, r->thick, m);
    const dim3 g2((r->w + 255) / 256, r->h);
    const float Fy = cam->proj[0], Fx = cam->proj[5];  // the reference's names: Fy = P[0][0], Fx = P[1][1]
    float* a = r->z0;
    float* b = r->z1;
    for (int it = 0; it < cam->smooth_iterations; ++it) {
        k_smooth<<<g2, 256, 0, st>>>(a, b, r->w, r->h, Fx, Fy);
        float* t = a; a = b; b = t;
    }
    r->zfinal = a;
    k_normals<<<g2, 256, 0, st>>>(a, r->normal, r->w, r->h, Fx, Fy);
    k_room<<<g2, 256, 0, st>>>(c, r->room);
    k_shade<<<g2, 256, 0, st>>>(c, a, r->thick, r->normal, r->room, r->color);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return rfail(PBF_ERR_CUDA, cudaGetErrorString(e));
    r->last = st;
    return PBF_OK;
}

}  // namespace

extern "C" {

int pbf_render_create(int width, int height, pbf_render** out) {
    if (!out) return rfail(PBF_ERR_INVALID, "null argument");
    *out = nullptr;
    if (width <= 0 || height <= 0 || width > 16384 || height > 16384)
        return rfail(PBF_ERR_INVALID, "width and height must lie in [1, 16384]");
    pbf_render* r = new pbf_render();
    r->w = width;
    r->h = height;
    const size_t m = (size_t)width * height;
    cudaError_t e = cudaSuccess;
    e = e ? e : cudaMalloc((void**)&r->depth, m * 8);
    e = e ? e : cudaMalloc((void**)&r->thick64, m * 8);
    e = e ? e : cudaMalloc((void**)&r->zraw, m * 4);
    e = e ? e : cudaMalloc((void**)&r->z0, m * 4);
    e = e ? e : cudaMalloc((void**)&r->z1, m * 4);
    e = e ? e : cudaMalloc((void**)&r->thick, m * 4);
    e = e ? e : cudaMalloc((void**)&r->normal, m * 16);
    e = e ? e : cudaMalloc((void**)&r->room, m * 16);
    e = e ? e : cudaMalloc((void**)&r->color, m * 16);
    if (e != cudaSuccess) {
        rfree(r);
        delete r;
        return rfail(PBF_ERR_ALLOC, "cudaMalloc of the render images failed");
    }
    r->zfinal = r->z0;
    *out = r;
    return PBF_OK;
}

int pbf_render_destroy(pbf_render* r) {
    if (!r) return PBF_OK;
    cudaStreamSynchronize(r->last);
    rfree(r);
    delete r;
    return PBF_OK;
}

int pbf_render_frame(pbf_render* r, const float* d_pos, int n, int stride, const pbf_camera* cam, void* stream) {
    return render_points(r, d_pos, n, stride, cam, (cudaStream_t)stream);
}

int pbf_render_frame_solver(pbf_render* r, pbf_solver* s, const pbf_camera* cam, void* stream) {
    const float4* x = nullptr;
    int n = 0;
    const int rc = pbf::solver_positions(s, &x, &n);
    if (rc) return rc;
    return render_points(r, reinterpret_cast<const float*>(x), n, 4, cam, (cudaStream_t)stream);
}

int pbf_render_read(pbf_render* r, int image, float* host, size_t count) {
    if (!r || !host) return rfail(PBF_ERR_INVALID, "null argument");
    const size_t m = (size_t)r->w * r->h;
    const void* src = nullptr;
    size_t floats = m;
    switch (image) {
        case PBF_IMAGE_DEPTH_RAW: src = r->zraw; break;
        case PBF_IMAGE_DEPTH: src = r->zfinal; break;
        case PBF_IMAGE_THICKNESS: src = r->thick; break;
        case PBF_IMAGE_NORMAL: src = r->normal; floats = 4 * m; break;
        case PBF_IMAGE_ROOM: src = r->room; floats = 4 * m; break;
        case PBF_IMAGE_COLOR: src = r->color; floats = 4 * m; break;
        default: return rfail(PBF_ERR_INVALID, "unknown image id");
    }
    if (count < floats) return rfail(PBF_ERR_INVALID, "host buffer too small for the image");
    if (cudaStreamSynchronize(r->last) != cudaSuccess || cudaMemcpy(host, src, floats * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        return rfail(PBF_ERR_CUDA, "reading the image failed");
    return PBF_OK;
}

}  // extern "C"
