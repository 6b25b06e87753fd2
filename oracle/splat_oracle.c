/*
 * CPU restatement of the reference pinhole 3DGS rasterizer (the oracle).
 * TEST INFRASTRUCTURE ONLY — see splat_oracle.h for the reference map.
 */
#include "splat_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define TILE 16

/* Gaussian exponent with the reference's rounding sequence
 * (geometry.cuh:26-33): -0.5 * fma(dx, a dx, (c dy) dy) - (b dx) dy. */
static float gpower(const float* co, float dx, float dy) {
    const float xx = co[0] * dx;
    const float yy = (co[2] * dy) * dy;
    const float xy = (co[1] * dx) * dy;
    return -0.5f * fmaf(dx, xx, yy) - xy;
}
#define ALPHA_FLOOR (1.0f / 255.0f)
#define T_FLOOR 1.0e-4f

static const float SH0 = 0.28209479177387814f;
static const float SH1 = 0.4886025119029199f;
static const float SH2[5] = {1.0925484305920792f, -1.0925484305920792f, 0.31539156525252005f,
                             -1.0925484305920792f, 0.5462742152960396f};
static const float SH3[7] = {-0.5900435899266435f, 2.890611442640554f, -0.4570457994644658f,
                             0.3731763325901154f, -0.4570457994644658f, 1.445305721320277f,
                             -0.5900435899266435f};


/* ---------------------------------------------------------------- algebra */
typedef struct { float m[3][3]; } m3;

static m3 mul3(const m3* a, const m3* b) {
    m3 o;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            o.m[i][j] = a->m[i][0] * b->m[0][j] + a->m[i][1] * b->m[1][j] + a->m[i][2] * b->m[2][j];
    return o;
}

static m3 tr3(const m3* a) {
    m3 o;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            o.m[i][j] = a->m[j][i];
    return o;
}

/* rotation rows of a scalar-first unit quaternion (matrix.cuh:125-139) */
static m3 quat_rows(const float q[4]) {
    const float r = q[0], x = q[1], y = q[2], z = q[3];
    m3 o;
    o.m[0][0] = 1.f - 2.f * (y * y + z * z);
    o.m[0][1] = 2.f * (x * y + r * z);
    o.m[0][2] = 2.f * (x * z - r * y);
    o.m[1][0] = 2.f * (x * y - r * z);
    o.m[1][1] = 1.f - 2.f * (x * x + z * z);
    o.m[1][2] = 2.f * (y * z + r * x);
    o.m[2][0] = 2.f * (x * z + r * y);
    o.m[2][1] = 2.f * (y * z - r * x);
    o.m[2][2] = 1.f - 2.f * (x * x + y * y);
    return o;
}

static void to_cam(const float* v, const float p[3], float t[3]) {
    t[0] = v[0] * p[0] + v[4] * p[1] + v[8] * p[2] + v[12];
    t[1] = v[1] * p[0] + v[5] * p[1] + v[9] * p[2] + v[13];
    t[2] = v[2] * p[0] + v[6] * p[1] + v[10] * p[2] + v[14];
}

static m3 view_rows(const float* v) {
    m3 w;
    w.m[0][0] = v[0]; w.m[0][1] = v[1]; w.m[0][2] = v[2];
    w.m[1][0] = v[4]; w.m[1][1] = v[5]; w.m[1][2] = v[6];
    w.m[2][0] = v[8]; w.m[2][1] = v[9]; w.m[2][2] = v[10];
    return w;
}

/* ------------------------------------------------------------- activation */
typedef struct {
    float scale[3], raw_scale[3], rot[4], opacity;
} activated;

static activated activate(const float* ls, const float* q, float logit) {
    activated a;
    float ratio = 1.f;
    for (int k = 0; k < 3; ++k) {
        const float v = expf(ls[k]);
        a.raw_scale[k] = v;
        a.scale[k] = sqrtf(v * v);
        ratio *= v / a.scale[k];
    }
    float nn = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    if (nn < 1e-20f) nn = 1e-20f;
    const float inv = 1.f / sqrtf(nn);
    for (int k = 0; k < 4; ++k)
        a.rot[k] = q[k] * inv;
    a.opacity = (1.f / (1.f + expf(-logit))) * ratio;
    return a;
}

/* ------------------------------------------------------------- projection */
typedef struct {
    float a, b, c, coef;
} cov2d;

/* EWA screen covariance with the 1.3 tan(fov) clamp (geometry.cuh:127-253) */
static cov2d project_cov(const float mean[3], const orc_camera* K, const float s[3],
                         const float q[4]) {
    float t[3];
    to_cam(K->view, mean, t);
    const float tfx = (float)K->width / (2.f * K->fx), tfy = (float)K->height / (2.f * K->fy);
    const float lx = 1.3f * tfx, ly = 1.3f * tfy;
    float u = t[0] / t[2], v = t[1] / t[2];
    t[0] = fminf(lx, fmaxf(-lx, u)) * t[2];
    t[1] = fminf(ly, fmaxf(-ly, v)) * t[2];
    m3 J;
    memset(&J, 0, sizeof J);
    J.m[0][0] = K->fx / t[2];
    J.m[1][1] = K->fy / t[2];
    J.m[2][0] = -(K->fx * t[0]) / (t[2] * t[2]);
    J.m[2][1] = -(K->fy * t[1]) / (t[2] * t[2]);
    const m3 W = view_rows(K->view);
    const m3 T = mul3(&W, &J);
    m3 S;
    memset(&S, 0, sizeof S);
    for (int k = 0; k < 3; ++k)
        S.m[k][k] = K->scale_modifier * s[k];
    const m3 R = quat_rows(q);
    const m3 SR = mul3(&S, &R);
    const m3 M = mul3(&SR, &T);
    const m3 Mt = tr3(&M);
    const m3 cov = mul3(&Mt, &M);
    cov2d o;
    o.a = cov.m[0][0] + K->kernel_size;
    o.b = cov.m[0][1];
    o.c = cov.m[1][1] + K->kernel_size;
    const float det0 = fmaxf(1.0e-6f, cov.m[0][0] * cov.m[1][1] - cov.m[0][1] * cov.m[0][1]);
    const float det1 = fmaxf(1.0e-6f, o.a * o.c - o.b * o.b);
    o.coef = K->compensate_2d ? sqrtf(det0 / det1) : 1.f;
    return o;
}

typedef struct {
    float q, lambda, da, db, dc;
} capinfo;

/* screen covariance cap lambda_max <= min(1024,W,H)^2/8 (footprint.cuh:14-27) */
static capinfo cov_cap(float a, float b, float c, int w, int h) {
    const float half = .5f * (a - c);
    const float radius = hypotf(half, b);
    const float lambda = .5f * a + .5f * c + radius;
    const float limit = fminf(1024.f, (float)(w < h ? w : h));
    const float variance = .125f * limit * limit;
    capinfo r = {1.f, lambda, 0.f, 0.f, 0.f};
    if (!(lambda > variance) || !isfinite(lambda))
        return r;
    const float hh = radius > 0.f ? half / radius : 0.f;
    r.q = variance / lambda;
    r.da = .5f + .5f * hh;
    r.db = radius > 0.f ? b / radius : 0.f;
    r.dc = .5f - .5f * hh;
    return r;
}

/* -------------------------------------------------------------- tile walk */
/* AccuTile walk along the shorter axis (tiles.cuh:115-179). If keys != NULL
 * instances are written; returns the count. */
static unsigned walk(float mx, float my, const float co[4], int gx, int gy, uint64_t* keys,
                     uint32_t* values, uint32_t gid, uint32_t depth_bits) {
    const float a = co[0], b = co[1], c = co[2];
    const float det = a * c - b * b;
    if (!(a > 0.f && c > 0.f) || !(co[3] >= 1.f / 255.f) || !(det > 0.f))
        return 0;
    const float th = 2.f * logf(co[3] * 255.f);
    if (!(th >= 0.f))
        return 0;
    const float ex = sqrtf(th * c / det), ey = sqrtf(th * a / det);
    const int along_x = (2.f * ex) / TILE <= (2.f * ey) / TILE;
    const float cu = along_x ? mx : my, cv = along_x ? my : mx;
    const float au = along_x ? a : c, av = along_x ? c : a;
    const int gu = along_x ? gx : gy, gv = along_x ? gy : gx;
    const float eu = sqrtf(th * av / det), ev = sqrtf(th * au / det);
    int umin = (int)floorf((cu - eu) / TILE), umax = (int)floorf((cu + eu) / TILE) + 1;
    if (umin > gu) umin = gu;
    if (umin < 0) umin = 0;
    if (umax > gu) umax = gu;
    if (umin >= umax)
        return 0;
    const float avmin = cu + b * ev / au, avmax = cu - b * ev / au;
    unsigned count = 0;
    for (int tu = umin; tu < umax; ++tu) {
        const float s0 = fmaxf(cu - eu, tu * (float)TILE), s1 = fminf(cu + eu, (tu + 1) * (float)TILE);
        const float d0 = s0 - cu, d1 = s1 - cu;
        const float r0 = sqrtf(fmaxf(0.f, av * th - det * d0 * d0));
        const float r1 = sqrtf(fmaxf(0.f, av * th - det * d1 * d1));
        const float lo = (avmin >= s0 && avmin <= s1) ? cv - ev
                                                       : fminf(cv + (-b * d0 - r0) / av, cv + (-b * d1 - r1) / av);
        const float hi = (avmax >= s0 && avmax <= s1) ? cv + ev
                                                       : fmaxf(cv + (-b * d0 + r0) / av, cv + (-b * d1 + r1) / av);
        int vmin = (int)floorf(lo / TILE), vmax = (int)floorf(hi / TILE) + 1;
        if (vmin > gv) vmin = gv;
        if (vmin < 0) vmin = 0;
        if (vmax > gv) vmax = gv;
        for (int tv = vmin; tv < vmax; ++tv) {
            if (keys) {
                const int tx = along_x ? tu : tv, ty = along_x ? tv : tu;
                const uint64_t tile = (uint64_t)ty * (uint64_t)gx + (uint64_t)tx;
                keys[count] = (tile << 32) | depth_bits;
                values[count] = gid;
            }
            ++count;
        }
    }
    return count;
}

/* --------------------------------------------------------------------- SH */
static void sh_basis(const float d[3], int degree, float w[16]) {
    const float x = d[0], y = d[1], z = d[2];
    for (int k = 0; k < 16; ++k) w[k] = 0.f;
    w[0] = SH0;
    if (degree > 0) {
        w[1] = -SH1 * y;
        w[2] = SH1 * z;
        w[3] = -SH1 * x;
    }
    if (degree > 1) {
        const float xx = x * x, yy = y * y, zz = z * z;
        const float q2[5] = {x * y, y * z, 2.f * zz - xx - yy, x * z, xx - yy};
        for (int k = 0; k < 5; ++k) w[4 + k] = SH2[k] * q2[k];
        if (degree > 2) {
            const float q3[7] = {y * (3.f * xx - yy), x * y * z, y * (4.f * zz - xx - yy),
                                 z * (2.f * zz - 3.f * xx - 3.f * yy), x * (4.f * zz - xx - yy),
                                 z * (xx - yy), x * (xx - 3.f * yy)};
            for (int k = 0; k < 7; ++k) w[9 + k] = SH3[k] * q3[k];
        }
    }
}

/* Derivatives of the basis functions with respect to the unit direction. */
static void sh_basis_grad(const float d[3], int degree, float gx[16], float gy[16], float gz[16]) {
    const float x = d[0], y = d[1], z = d[2];
    for (int k = 0; k < 16; ++k) gx[k] = gy[k] = gz[k] = 0.f;
    if (degree > 0) {
        gy[1] = -SH1;
        gz[2] = SH1;
        gx[3] = -SH1;
    }
    if (degree > 1) {
        const float dx[5] = {y, 0.f, -2.f * x, z, 2.f * x};
        const float dy[5] = {x, z, -2.f * y, 0.f, -2.f * y};
        const float dz[5] = {0.f, y, 4.f * z, x, 0.f};
        for (int k = 0; k < 5; ++k) {
            gx[4 + k] = SH2[k] * dx[k];
            gy[4 + k] = SH2[k] * dy[k];
            gz[4 + k] = SH2[k] * dz[k];
        }
        if (degree > 2) {
            const float xx = x * x, yy = y * y, zz = z * z;
            const float dx3[7] = {6.f * x * y, y * z, -2.f * x * y, -6.f * x * z,
                                  -3.f * xx + 4.f * zz - yy, 2.f * x * z, 3.f * (xx - yy)};
            const float dy3[7] = {3.f * (xx - yy), x * z, -3.f * yy + 4.f * zz - xx, -6.f * y * z,
                                  -2.f * x * y, -2.f * y * z, -6.f * x * y};
            const float dz3[7] = {0.f, x * y, 8.f * y * z, 3.f * (2.f * zz - xx - yy), 8.f * x * z,
                                  xx - yy, 0.f};
            for (int k = 0; k < 7; ++k) {
                gx[9 + k] = SH3[k] * dx3[k];
                gy[9 + k] = SH3[k] * dy3[k];
                gz[9 + k] = SH3[k] * dz3[k];
            }
        }
    }
}

static void view_dir(const float* pos, const float* cam, float d[3], float* inv_len) {
    const float v[3] = {pos[0] - cam[0], pos[1] - cam[1], pos[2] - cam[2]};
    const float inv = 1.f / sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    for (int k = 0; k < 3; ++k) d[k] = v[k] * inv;
    *inv_len = inv;
}

/* ------------------------------------------------------------- preprocess */
void orc_preprocess(int n, const float* means, const float* log_scales, const float* quats,
                    const float* logits, const float* sh, int sh_degree, int sh_bases,
                    const orc_camera* K, float* mean2d, float* conic, float* rgb, uint8_t* clamp,
                    float* depth, int* radii, uint32_t* touched, int32_t* bounds, int begin,
                    int end) {
    const int gx = (K->width + TILE - 1) / TILE, gy = (K->height + TILE - 1) / TILE;
    (void)n;
    for (int i = begin; i < end; ++i) {
        touched[i] = 0;
        radii[i] = 0;
        const float* m = means + 3 * i;
        float t[3];
        to_cam(K->view, m, t);
        if (!(t[2] > K->near_plane))
            continue;
        const activated act = activate(log_scales + 3 * i, quats + 4 * i, logits[i]);
        cov2d cv = project_cov(m, K, act.scale, act.rot);
        const capinfo cap = cov_cap(cv.a, cv.b, cv.c, K->width, K->height);
        if (cap.q < 1.f) {
            cv.a *= cap.q;
            cv.b *= cap.q;
            cv.c *= cap.q;
        }
        const float iz = 1.f / t[2];
        const float px = t[0] * iz * K->fx + K->cx, py = t[1] * iz * K->fy + K->cy;
        const float det = cv.a * cv.c - cv.b * cv.b;
        if (det == 0.f)
            continue;
        const float di = 1.f / det;
        const float co[4] = {cv.c * di, -cv.b * di, cv.a * di, act.opacity * cv.coef};
        const float mid = 0.5f * (cv.a + cv.c);
        const float root = sqrtf(fmaxf(0.1f, mid * mid - det));
        const float radius = ceilf(3.f * sqrtf(fmaxf(mid + root, mid - root)));
        const unsigned cnt = walk(px, py, co, gx, gy, NULL, NULL, 0, 0);
        if (cnt == 0)
            continue;
        float d[3], inv;
        view_dir(m, K->center, d, &inv);
        float w[16];
        sh_basis(d, sh_degree, w);
        uint8_t cb = 0;
        for (int ch = 0; ch < 3; ++ch) {
            float acc = 0.f;
            for (int k = 0; k < (sh_degree + 1) * (sh_degree + 1); ++k)
                acc += w[k] * sh[((size_t)i * sh_bases + k) * 3 + ch];
            acc += 0.5f;
            if (acc < 0.f) cb |= (uint8_t)(1u << ch);
            rgb[3 * i + ch] = fmaxf(acc, 0.f);
        }
        clamp[i] = cb;
        mean2d[2 * i] = px;
        mean2d[2 * i + 1] = py;
        for (int k = 0; k < 4; ++k) conic[4 * i + k] = co[k];
        depth[i] = sqrtf(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
        radii[i] = (int)radius;
        touched[i] = cnt;
        const float th = 2.f * logf(co[3] * 255.f);
        const float ex = sqrtf(fmaxf(0.f, th * cv.a)), ey = sqrtf(fmaxf(0.f, th * cv.c));
        bounds[4 * i + 0] = (int32_t)fmaxf(0.f, floorf(px - ex));
        bounds[4 * i + 1] = (int32_t)fmaxf(0.f, floorf(px + ex) + 1.f);
        bounds[4 * i + 2] = (int32_t)fmaxf(0.f, floorf(py - ey));
        bounds[4 * i + 3] = (int32_t)fmaxf(0.f, floorf(py + ey) + 1.f);
    }
}

void orc_emit(int n, const float* mean2d, const float* conic, const float* depth,
              const uint32_t* touched, const uint64_t* offsets, int gx, int gy, uint64_t* keys,
              uint32_t* values) {
    for (int i = 0; i < n; ++i) {
        if (!touched[i])
            continue;
        uint32_t bits;
        memcpy(&bits, &depth[i], 4);
        walk(mean2d[2 * i], mean2d[2 * i + 1], conic + 4 * i, gx, gy, keys + offsets[i],
             values + offsets[i], (uint32_t)i, bits);
    }
}

/* ------------------------------------------------------------- composite */
void orc_composite(int tiles, const uint32_t* ranges, const uint32_t* order, const float* mean2d,
                   const float* conic, const float* rgb, const orc_camera* K, const float* bg,
                   int use_double, double* color, double* alpha, double* T_final, uint32_t* last,
                   float* visibility, int tile_begin, int tile_end) {
    const int gx = (K->width + TILE - 1) / TILE;
    const size_t P = (size_t)K->width * K->height;
    (void)tiles;
    for (int tile = tile_begin; tile < tile_end; ++tile) {
        const int tx = tile % gx, ty = tile / gx;
        const uint32_t r0 = ranges[2 * tile], r1 = ranges[2 * tile + 1];
        for (int ly = 0; ly < TILE; ++ly)
            for (int lx = 0; lx < TILE; ++lx) {
                const int px = tx * TILE + lx, py = ty * TILE + ly;
                if (px >= K->width || py >= K->height)
                    continue;
                const size_t pid = (size_t)py * K->width + px;
                double T = 1.0, c[3] = {0, 0, 0};
                float Tf = 1.f, cf[3] = {0.f, 0.f, 0.f};
                uint32_t lastc = 0;
                for (uint32_t k = r0; k < r1; ++k) {
                    const uint32_t g = order[k];
                    const float* co = conic + 4 * g;
                    const float dx = mean2d[2 * g] - (float)px, dy = mean2d[2 * g + 1] - (float)py;
                    const float power = gpower(co, dx, dy);
                    if (power > 0.f)
                        continue;
                    const float a = fminf(K->alpha_clip, co[3] * expf(power));
                    if (a < ALPHA_FLOOR)
                        continue;
                    if (use_double) {
                        const double tt = T * (1.0 - a);
                        if (tt < T_FLOOR) break;
                        for (int ch = 0; ch < 3; ++ch) c[ch] += rgb[3 * g + ch] * (double)a * T;
                        T = tt;
                    } else {
                        const float tt = Tf * (1.f - a);
                        if (tt < T_FLOOR) break;
                        for (int ch = 0; ch < 3; ++ch) cf[ch] += rgb[3 * g + ch] * (a * Tf);
                        Tf = tt;
                    }
                    lastc = k - r0 + 1;
                    if (visibility) visibility[g] = 1.f;
                }
                if (!use_double) {
                    T = Tf;
                    for (int ch = 0; ch < 3; ++ch) c[ch] = cf[ch];
                }
                for (int ch = 0; ch < 3; ++ch) color[ch * P + pid] = c[ch] + T * bg[ch];
                alpha[pid] = 1.0 - T;
                T_final[pid] = T;
                last[pid] = lastc;
            }
    }
}

/* ----------------------------------------------------- geometry channels */
/* Ray plane and footprint normal (geometry.cuh:255-275, pinhole branch,
 * scale/rotation form), for visible Gaussians (radii[i] > 0): plane[4i..] =
 * (d depth / d dx, d depth / d dy, distance of the centre, 1/sigma along the
 * ray at the peak), normal[3i..] = unit camera-space normal. */
void orc_geometry(int n, const float* means, const float* log_scales, const float* quats,
                  const float* logits, const orc_camera* K, const int* radii, float* plane,
                  float* normal, int begin, int end) {
    (void)n;
    for (int i = begin; i < end; ++i) {
        if (radii[i] <= 0)
            continue;
        const activated act = activate(log_scales + 3 * i, quats + 4 * i, logits[i]);
        float t[3];
        to_cam(K->view, means + 3 * i, t);
        const float tc = sqrtf(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
        const float tfx = (float)K->width / (2.f * K->fx), tfy = (float)K->height / (2.f * K->fy);
        const float lx = 1.3f * tfx, ly = 1.3f * tfy;
        float u = t[0] / t[2], v = t[1] / t[2];
        t[0] = fminf(lx, fmaxf(-lx, u)) * t[2];
        t[1] = fminf(ly, fmaxf(-ly, v)) * t[2];
        u = t[0] / t[2];
        v = t[1] / t[2];
        const m3 W = view_rows(K->view);
        m3 Si;
        memset(&Si, 0, sizeof Si);
        for (int k = 0; k < 3; ++k)
            Si.m[k][k] = 1.f / (K->scale_modifier * act.scale[k]);
        const m3 R = quat_rows(act.rot);
        const m3 SR = mul3(&Si, &R);
        const m3 Mi = mul3(&SR, &W);
        const m3 Mit = tr3(&Mi);
        const m3 ci = mul3(&Mit, &Mi); /* inverse covariance in camera space */
        const float uvh[3] = {u, v, 1.f};
        float um[3];
        for (int r = 0; r < 3; ++r)
            um[r] = ci.m[r][0] * uvh[0] + ci.m[r][1] * uvh[1] + ci.m[r][2] * uvh[2];
        const float u2 = u * u, v2 = v * v;
        const float l = sqrtf(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
        const float vb = um[0] * uvh[0] + um[1] * uvh[1] + um[2] * uvh[2];
        const float rl2 = u2 + v2 + 1.f;
        const float fn = l / rl2;
        const float q[3] = {um[0] / vb, um[1] / vb, um[2] / vb};
        /* rows of the inverse peak Jacobian: (v^2+1, -uv, -u), (-uv, u^2+1, -v) */
        const float pl0 = (v2 + 1.f) * q[0] + -(u * v) * q[1] + -u * q[2];
        const float pl1 = -(u * v) * q[0] + (u2 + 1.f) * q[1] + -v * q[2];
        plane[4 * i + 0] = pl0 * fn / K->fx;
        plane[4 * i + 1] = pl1 * fn / K->fy;
        plane[4 * i + 2] = tc;
        plane[4 * i + 3] = sqrtf(vb / rl2);
        const float rn[3] = {-pl0 * fn, -pl1 * fn, -1.f};
        const float iz = 1.f / t[2];
        const float cn[3] = {iz * rn[0] + (t[0] / l) * rn[2], iz * rn[1] + (t[1] / l) * rn[2],
                             (-t[0] * iz * iz) * rn[0] + (-t[1] * iz * iz) * rn[1] +
                                 (t[2] / l) * rn[2]};
        const float inv = 1.f / sqrtf(cn[0] * cn[0] + cn[1] * cn[1] + cn[2] * cn[2]);
        for (int k = 0; k < 3; ++k)
            normal[3 * i + k] = cn[k] * inv;
    }
}

#define DEPTH_SPLIT 8
#define DEPTH_REFINEMENTS 5
#define DEPTH_SEED_WINDOW 0.4f
#define DEPTH_MIN_T 0.45f

/* Median depth [P] (camera-space Z) and alpha-normalised normal [3P] of every
 * pixel of the tiles (render_forward.cu:341-525, blend_tile<GEOMETRY>): the
 * colour pass also accumulates the normal and the depth seed (plane depth of
 * the last Gaussian blended while T > 0.5); the bisection then brackets the
 * depth where the transmittance along the ray crosses 0.5 (8 probes in
 * +-0.4 around the seed, 5 refinements over the pixel's contributors) and
 * interpolates inside the final bracket. FP32. */
void orc_median_depth(int tiles, const uint32_t* ranges, const uint32_t* order,
                      const float* mean2d, const float* conic, const float* plane,
                      const float* normal, const orc_camera* K, float* depth_out,
                      float* normal_out, int tile_begin, int tile_end) {
    const int gx = (K->width + TILE - 1) / TILE;
    const size_t P = (size_t)K->width * K->height;
    (void)tiles;
    for (int tile = tile_begin; tile < tile_end; ++tile) {
        const int tx = tile % gx, ty = tile / gx;
        const uint32_t r0 = ranges[2 * tile], r1 = ranges[2 * tile + 1];
        for (int ly = 0; ly < TILE; ++ly)
            for (int lx = 0; lx < TILE; ++lx) {
                const int px = tx * TILE + lx, py = ty * TILE + ly;
                if (px >= K->width || py >= K->height)
                    continue;
                const size_t pid = (size_t)py * K->width + px;
                float T = 1.f, nacc[3] = {0.f, 0.f, 0.f}, seed = 0.f;
                uint32_t lastc = 0;
                for (uint32_t k = r0; k < r1; ++k) {
                    const uint32_t g = order[k];
                    const float* co = conic + 4 * g;
                    const float dx = mean2d[2 * g] - (float)px, dy = mean2d[2 * g + 1] - (float)py;
                    const float power = gpower(co, dx, dy);
                    if (power > 0.f)
                        continue;
                    const float a = fminf(K->alpha_clip, co[3] * expf(power));
                    if (a < ALPHA_FLOOR)
                        continue;
                    const float tt = T * (1.f - a);
                    if (tt < T_FLOOR)
                        break;
                    const float w = a * T;
                    const float* rp = plane + 4 * g;
                    const float td = rp[0] * dx + rp[1] * dy + rp[2];
                    for (int ch = 0; ch < 3; ++ch)
                        nacc[ch] += normal[3 * g + ch] * w;
                    seed = T > 0.5f ? td : seed;
                    T = tt;
                    lastc = k - r0 + 1;
                }
                float dmin = fmaxf(seed - DEPTH_SEED_WINDOW, 0.f);
                float dmax = fmaxf(seed + DEPTH_SEED_WINDOW, 0.f);
                int in_range = T <= DEPTH_MIN_T;
                float Tp[DEPTH_SPLIT + 1];
                for (int it = 0; it < DEPTH_REFINEMENTS; ++it) {
                    const int first = it == 0;
                    const int s0 = first ? 0 : 1, s1 = first ? DEPTH_SPLIT + 1 : DEPTH_SPLIT;
                    for (int s = s0; s < s1; ++s)
                        Tp[s] = 1.f;
                    const float interval = (dmax - dmin) * (1.f / (float)DEPTH_SPLIT);
                    for (uint32_t k = r0; in_range && k < r0 + lastc; ++k) {
                        const uint32_t g = order[k];
                        const float* co = conic + 4 * g;
                        const float dx = mean2d[2 * g] - (float)px,
                                    dy = mean2d[2 * g + 1] - (float)py;
                        const float power = gpower(co, dx, dy);
                        if (power > 0.f)
                            continue;
                        const float a = fminf(K->alpha_clip, co[3] * expf(power));
                        if (a < ALPHA_FLOOR)
                            continue;
                        const float* rp = plane + 4 * g;
                        const float tpk = rp[0] * dx + rp[1] * dy + rp[2];
                        const float rs = rp[3];
                        for (int s = s0; s < s1; ++s) {
                            const float ts = dmin + interval * (float)s;
                            const float dl = (ts - tpk) * rs;
                            const float gk = rs > 0.f ? expf(-0.5f * dl * dl) : 0.f;
                            const float omg = 1.f - a * gk;
                            Tp[s] *= (ts > tpk ? (1.f - a) : omg) * (1.f / sqrtf(omg));
                        }
                    }
                    if (first)
                        in_range = Tp[0] >= 0.5f && Tp[DEPTH_SPLIT] <= 0.5f && in_range;
                    int st = 0;
                    for (int s = 1; s < DEPTH_SPLIT; ++s)
                        st = Tp[s] >= 0.5f ? s : st;
                    dmax = dmin + (float)(st + 1) * interval;
                    dmin = dmin + (float)st * interval;
                    const float lo = Tp[st], hi = Tp[st + 1];
                    Tp[0] = lo;
                    Tp[DEPTH_SPLIT] = hi;
                }
                float wm = (Tp[0] - 0.5f) / (Tp[0] - Tp[DEPTH_SPLIT]);
                wm = wm != wm ? 0.f : fminf(fmaxf(wm, 0.f), 1.f); /* saturate, NaN -> 0 */
                const float median = in_range ? wm * dmax + (1.f - wm) * dmin : 0.f;
                const float x = ((float)px - K->cx) / K->fx, y = ((float)py - K->cy) / K->fy;
                depth_out[pid] = median * (1.f / sqrtf(x * x + y * y + 1.f));
                const float len = 1.f - T;
                for (int ch = 0; ch < 3; ++ch)
                    normal_out[ch * P + pid] = lastc ? nacc[ch] / len : 0.f;
            }
    }
}

/* ---------------------------------------------------------- composite bwd */
void orc_composite_backward(int tiles, const uint32_t* ranges, const uint32_t* order,
                            const float* mean2d, const float* conic, const float* rgb,
                            const orc_camera* K, const float* bg, const double* T_final,
                            const uint32_t* last, const float* dL_color, const float* dL_alpha,
                            int n, double* grad12, int tile_begin, int tile_end) {
    (void)n;
    (void)tiles;
    const int gx = (K->width + TILE - 1) / TILE;
    const size_t P = (size_t)K->width * K->height;
    for (int tile = tile_begin; tile < tile_end; ++tile) {
        const int tx = tile % gx, ty = tile / gx;
        const uint32_t r0 = ranges[2 * tile];
        for (int ly = 0; ly < TILE; ++ly)
            for (int lx = 0; lx < TILE; ++lx) {
                const int px = tx * TILE + lx, py = ty * TILE + ly;
                if (px >= K->width || py >= K->height)
                    continue;
                const size_t pid = (size_t)py * K->width + px;
                const double g[3] = {dL_color[pid], dL_color[P + pid], dL_color[2 * P + pid]};
                const double Tf = T_final[pid];
                const double dfin = bg[0] * g[0] + bg[1] * g[1] + bg[2] * g[2] -
                                    (dL_alpha ? dL_alpha[pid] : 0.0);
                const double refine_scale = 1.0 / fmax(1.0 - Tf, 1.0e-5);
                double T = Tf, sdot = 0.0;
                for (int k = (int)last[pid] - 1; k >= 0; --k) {
                    const uint32_t gid = order[r0 + k];
                    const float* co = conic + 4 * gid;
                    const float dx = mean2d[2 * gid] - (float)px, dy = mean2d[2 * gid + 1] - (float)py;
                    const float power = gpower(co, dx, dy);
                    if (power > 0.f)
                        continue;
                    const double G = exp((double)power);
                    const double a = fmin(K->alpha_clip, co[3] * G);
                    if (a < ALPHA_FLOOR)
                        continue;
                    T = T / (1.0 - a);
                    const double w = a * T;
                    const double* cc = NULL;
                    (void)cc;
                    const double cdot = rgb[3 * gid] * g[0] + rgb[3 * gid + 1] * g[1] + rgb[3 * gid + 2] * g[2];
                    const double dLda = T * cdot - (sdot + Tf * dfin) / (1.0 - a);
                    sdot += w * cdot;
                    const double dLdG = co[3] * dLda;
                    const double gdx = G * dx, gdy = G * dy;
                    const double dmx = dLdG * (-gdx * co[0] - gdy * co[1]);
                    const double dmy = dLdG * (-gdy * co[2] - gdx * co[1]);
                    double v[12] = {-0.5 * gdx * dx * dLdG, -0.5 * gdx * dy * dLdG,
                                    -0.5 * gdy * dy * dLdG, G * dLda, dmx, dmy,
                                    sqrt(dmx * K->width * dmx * K->width + dmy * K->height * dmy * K->height) * refine_scale,
                                    0.0, w * g[0], w * g[1], w * g[2], 0.0};
                    for (int q = 0; q < 12; ++q)
                        grad12[12 * (size_t)gid + q] += v[q];
                }
            }
    }
}

/* ----------------------------------------------------------- gaussian bwd */
void orc_gaussian_backward(int n, const float* means, const float* log_scales,
                           const float* quats, const float* logits, const float* sh,
                           int sh_degree, int sh_bases, const orc_camera* K, const int* radii,
                           const uint8_t* clamp, const double* grad12, int activated_out,
                           double* g_means, double* g_scales, double* g_rots, double* g_opac,
                           double* g_sh, int begin, int end) {
    (void)n;
    for (int i = begin; i < end; ++i) {
        if (radii[i] <= 0)
            continue;
        const double* G = grad12 + 12 * (size_t)i;
        const float* mean = means + 3 * i;
        const activated act = activate(log_scales + 3 * i, quats + 4 * i, logits[i]);
        /* forward quantities in double */
        float tf[3];
        to_cam(K->view, mean, tf);
        double t[3] = {tf[0], tf[1], tf[2]};
        const double fx = K->fx, fy = K->fy;
        const double lx = 1.3 * ((double)K->width / (2.0 * fx)), ly = 1.3 * ((double)K->height / (2.0 * fy));
        const double u0 = t[0] / t[2], v0 = t[1] / t[2];
        const double xm = (u0 < -lx || u0 > lx) ? 0.0 : 1.0, ym = (v0 < -ly || v0 > ly) ? 0.0 : 1.0;
        t[0] = fmin(lx, fmax(-lx, u0)) * t[2];
        t[1] = fmin(ly, fmax(-ly, v0)) * t[2];
        double J[3][2] = {{fx / t[2], 0.0}, {0.0, fy / t[2]},
                          {-(fx * t[0]) / (t[2] * t[2]), -(fy * t[1]) / (t[2] * t[2])}};
        double W[3][3];
        const float* v = K->view;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) W[r][c] = v[4 * r + c];
        /* A = d(px)/d(world) column 0 of T = W J, B = column 1 */
        double A[3], B[3];
        for (int r = 0; r < 3; ++r) {
            A[r] = W[r][0] * J[0][0] + W[r][1] * J[1][0] + W[r][2] * J[2][0];
            B[r] = W[r][0] * J[0][1] + W[r][1] * J[1][1] + W[r][2] * J[2][1];
        }
        double R[3][3];
        {
            const m3 Rf = quat_rows(act.rot);
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) R[r][c] = Rf.m[r][c];
        }
        const double sm = K->scale_modifier;
        double s[3] = {sm * act.scale[0], sm * act.scale[1], sm * act.scale[2]};
        double SR[3][3], V[3][3];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) SR[r][c] = s[r] * R[r][c];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c)
                V[r][c] = SR[0][r] * SR[0][c] + SR[1][r] * SR[1][c] + SR[2][r] * SR[2][c];
        double ca = 0, cb = 0, cc = 0;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                ca += A[r] * V[r][c] * A[c];
                cb += A[r] * V[r][c] * B[c];
                cc += B[r] * V[r][c] * B[c];
            }
        const double ks = K->kernel_size;
        const double det0 = fmax(1e-6, ca * cc - cb * cb);
        const double a = ca + ks, b = cb, c = cc + ks;
        const double det1 = fmax(1e-6, a * c - b * b);
        const double coef = K->compensate_2d ? sqrt(det0 / det1) : 1.0;
        /* conic adjoint (with cap) */
        const double dco[4] = {G[0], G[1], G[2], G[3]};
        const double den = a * c - b * b;
        const double den2 = 1.0 / (den * den + 1.0e-7);
        double da = den2 * (-c * c * dco[0] + 2.0 * b * c * dco[1] + (den - a * c) * dco[2]);
        double dc = den2 * (-a * a * dco[2] + 2.0 * a * b * dco[1] + (den - a * c) * dco[0]);
        double db = den2 * 2.0 * (b * c * dco[0] - (den + 2.0 * b * b) * dco[1] + a * b * dco[2]);
        const capinfo cap = cov_cap((float)a, (float)b, (float)c, K->width, K->height);
        if (cap.q < 1.f) {
            const double x = a * cap.q, y = b * cap.q, z = c * cap.q;
            const double dt = x * z - y * y;
            const double uu = z / dt, vv = -y / dt, ww = x / dt;
            const double ga = -(uu * uu * dco[0] + 2.0 * uu * vv * dco[1] + vv * vv * dco[2]);
            const double gb = -2.0 * (uu * vv * dco[0] + (uu * ww + vv * vv) * dco[1] + vv * ww * dco[2]);
            const double gc = -(vv * vv * dco[0] + 2.0 * vv * ww * dco[1] + ww * ww * dco[2]);
            const double pull = (ga * a + gb * b + gc * c) / cap.lambda;
            da = cap.q * (ga - pull * cap.da);
            db = cap.q * (gb - pull * cap.db);
            dc = cap.q * (gc - pull * cap.dc);
        }
        const double d_opac = dco[3] * coef;
        /* dL/dV (symmetric), from cov2d = [A;B] V [A;B]^T */
        double gV[3][3];
        for (int r = 0; r < 3; ++r)
            for (int q = 0; q < 3; ++q)
                gV[r][q] = A[r] * A[q] * da + 0.5 * (A[r] * B[q] + B[r] * A[q]) * db + B[r] * B[q] * dc;
        /* V = SR^T SR -> dL/dSR = 2 SR gV */
        double dSR[3][3];
        for (int r = 0; r < 3; ++r)
            for (int q = 0; q < 3; ++q)
                dSR[r][q] = 2.0 * (SR[r][0] * gV[0][q] + SR[r][1] * gV[1][q] + SR[r][2] * gV[2][q]);
        double d_scale[3], Q[3][3];
        for (int r = 0; r < 3; ++r) {
            d_scale[r] = sm * (R[r][0] * dSR[r][0] + R[r][1] * dSR[r][1] + R[r][2] * dSR[r][2]);
            for (int q = 0; q < 3; ++q) Q[r][q] = s[r] * dSR[r][q];
        }
        const double qr = act.rot[0], qx = act.rot[1], qy = act.rot[2], qz = act.rot[3];
        double d_rot[4];
        d_rot[0] = 2 * qz * (Q[0][1] - Q[1][0]) + 2 * qy * (Q[2][0] - Q[0][2]) + 2 * qx * (Q[1][2] - Q[2][1]);
        d_rot[1] = 2 * qy * (Q[0][1] + Q[1][0]) + 2 * qz * (Q[0][2] + Q[2][0]) + 2 * qr * (Q[1][2] - Q[2][1]) - 4 * qx * (Q[2][2] + Q[1][1]);
        d_rot[2] = 2 * qx * (Q[0][1] + Q[1][0]) + 2 * qr * (Q[2][0] - Q[0][2]) + 2 * qz * (Q[1][2] + Q[2][1]) - 4 * qy * (Q[2][2] + Q[0][0]);
        d_rot[3] = 2 * qr * (Q[0][1] - Q[1][0]) + 2 * qx * (Q[0][2] + Q[2][0]) + 2 * qy * (Q[1][2] + Q[2][1]) - 4 * qz * (Q[1][1] + Q[0][0]);
        /* cov2d through T = W J: dL/dA, dL/dB, then J -> t */
        double dA[3] = {0, 0, 0}, dB[3] = {0, 0, 0};
        for (int r = 0; r < 3; ++r)
            for (int q = 0; q < 3; ++q) {
                dA[r] += 2.0 * V[r][q] * A[q] * da + V[r][q] * B[q] * db;
                dB[r] += 2.0 * V[r][q] * B[q] * dc + V[r][q] * A[q] * db;
            }
        /* A = W[:,0] J00 + W[:,2] J20 ; B = W[:,1] J11 + W[:,2] J21 */
        double dJ00 = 0, dJ20 = 0, dJ11 = 0, dJ21 = 0;
        for (int r = 0; r < 3; ++r) {
            dJ00 += W[r][0] * dA[r];
            dJ20 += W[r][2] * dA[r];
            dJ11 += W[r][1] * dB[r];
            dJ21 += W[r][2] * dB[r];
        }
        const double tz = 1.0 / t[2];
        const double dtx = xm * (-fx * tz * tz * dJ20);
        const double dty = ym * (-fy * tz * tz * dJ21);
        const double dtz = -fx * tz * tz * dJ00 - fy * tz * tz * dJ11 +
                           (1.0 + xm) * fx * t[0] * tz * tz * tz * dJ20 +
                           (1.0 + ym) * fy * t[1] * tz * tz * tz * dJ21;
        double dm[3];
        dm[0] = v[0] * dtx + v[1] * dty + v[2] * dtz;
        dm[1] = v[4] * dtx + v[5] * dty + v[6] * dtz;
        dm[2] = v[8] * dtx + v[9] * dty + v[10] * dtz;
        /* pixel centre */
        {
            const double rz = 1.0 / ((double)tf[2] + 1.0e-7);
            const double sx = tf[0] * rz, sy = tf[1] * rz;
            const double gxp = G[4], gyp = G[5];
            dm[0] += (fx * (v[0] - sx * v[2]) * gxp + fy * (v[1] - sy * v[2]) * gyp) * rz;
            dm[1] += (fx * (v[4] - sx * v[6]) * gxp + fy * (v[5] - sy * v[6]) * gyp) * rz;
            dm[2] += (fx * (v[8] - sx * v[10]) * gxp + fy * (v[9] - sy * v[10]) * gyp) * rz;
        }
        /* SH adjoint */
        if (sh) {
            float d[3], inv;
            view_dir(mean, K->center, d, &inv);
            float w[16], wx[16], wy[16], wz[16];
            sh_basis(d, sh_degree, w);
            sh_basis_grad(d, sh_degree, wx, wy, wz);
            double dl[3] = {G[8], G[9], G[10]};
            for (int ch = 0; ch < 3; ++ch)
                if (clamp[i] & (1u << ch)) dl[ch] = 0.0;
            const int nb = (sh_degree + 1) * (sh_degree + 1);
            double ddir[3] = {0, 0, 0};
            for (int k = 0; k < nb; ++k)
                for (int ch = 0; ch < 3; ++ch) {
                    if (g_sh) g_sh[((size_t)i * sh_bases + k) * 3 + ch] += w[k] * dl[ch];
                    const double cf = sh[((size_t)i * sh_bases + k) * 3 + ch];
                    ddir[0] += wx[k] * cf * dl[ch];
                    ddir[1] += wy[k] * cf * dl[ch];
                    ddir[2] += wz[k] * cf * dl[ch];
                }
            const double dot = d[0] * ddir[0] + d[1] * ddir[1] + d[2] * ddir[2];
            for (int k = 0; k < 3; ++k) dm[k] += (ddir[k] - d[k] * dot) * inv;
        }
        for (int k = 0; k < 3; ++k) g_means[3 * i + k] += dm[k];
        if (activated_out) {
            for (int k = 0; k < 3; ++k) g_scales[3 * i + k] += d_scale[k];
            for (int k = 0; k < 4; ++k) g_rots[4 * i + k] += d_rot[k];
            g_opac[i] += d_opac;
        } else {
            for (int k = 0; k < 3; ++k) {
                const double raw = act.raw_scale[k], sc = act.scale[k];
                g_scales[3 * i + k] += d_scale[k] * raw * raw / sc;
            }
            const float* q = quats + 4 * i;
            double nn = (double)q[0] * q[0] + (double)q[1] * q[1] + (double)q[2] * q[2] + (double)q[3] * q[3];
            if (nn < 1e-20) nn = 1e-20;
            const double inv = 1.0 / sqrt(nn);
            double qn[4], qdot = 0;
            for (int k = 0; k < 4; ++k) {
                qn[k] = q[k] * inv;
                qdot += qn[k] * d_rot[k];
            }
            for (int k = 0; k < 4; ++k) g_rots[4 * i + k] += inv * (d_rot[k] - qn[k] * qdot);
            const double sig = 1.0 / (1.0 + exp(-(double)logits[i]));
            g_opac[i] += d_opac * act.opacity * (1.0 - sig);
        }
    }
}

/* ------------------------------------------------------------------- Adam */
void orc_adam(float* p, const float* g, float* m, float* v, long n, float lr, float b1, float b2,
              float c1, float c2, float eps, float lo, float hi) {
    for (long i = 0; i < n; ++i) {
        const float prev = p[i], gr = g[i];
        if (!isfinite(prev) || !isfinite(gr)) {
            m[i] = v[i] = 0.f;
            p[i] = isfinite(prev) ? fminf(fmaxf(prev, lo), hi) : fminf(fmaxf(0.f, lo), hi);
            continue;
        }
        const float mm = b1 * m[i] + (1.f - b1) * gr;
        const float vv = b2 * v[i] + (1.f - b2) * gr * gr;
        if (!isfinite(mm) || !isfinite(vv)) {
            m[i] = v[i] = 0.f;
            p[i] = fminf(fmaxf(prev, lo), hi);
            continue;
        }
        m[i] = mm;
        v[i] = vv;
        const float cand = prev - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
        p[i] = fminf(fmaxf(isfinite(cand) ? cand : prev, lo), hi);
    }
}

/* ---------------------------------------------------- SH Adam (quantized) */
static float half_to_float(uint16_t h) {
    const uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
    uint32_t exp = (h >> 10) & 0x1fu, mant = h & 0x3ffu, bits;
    if (exp == 0) {
        if (mant == 0) {
            bits = sign;
        } else { /* subnormal */
            exp = 127 - 15 + 1;
            while (!(mant & 0x400u)) {
                mant <<= 1;
                --exp;
            }
            mant &= 0x3ffu;
            bits = sign | (exp << 23) | (mant << 13);
        }
    } else if (exp == 31) {
        bits = sign | 0x7f800000u | (mant << 13);
    } else {
        bits = sign | ((exp + 127 - 15) << 23) | (mant << 13);
    }
    float f;
    memcpy(&f, &bits, 4);
    return f;
}

static uint16_t float_to_half(float f) { /* round to nearest even */
    uint32_t x;
    memcpy(&x, &f, 4);
    const uint32_t sign = (x >> 16) & 0x8000u;
    const uint32_t absx = x & 0x7fffffffu;
    if (absx >= 0x7f800000u) /* inf / nan */
        return (uint16_t)(sign | 0x7c00u | (absx > 0x7f800000u ? 0x200u : 0u));
    if (absx >= 0x477ff000u) /* rounds to >= 65520: inf */
        return (uint16_t)(sign | 0x7c00u);
    if (absx < 0x38800000u) { /* subnormal half or zero */
        if (absx < 0x33000000u)
            return (uint16_t)sign;
        const uint32_t e = absx >> 23;
        uint32_t m = (absx & 0x7fffffu) | 0x800000u;
        /* value = m * 2^(e-150); half subnormal unit = 2^-24 */
        const int s = 126 - (int)e; /* right shift of m to units of 2^-24 */
        uint32_t q = m >> s;
        const uint32_t rem = m & ((1u << s) - 1u), halfway = 1u << (s - 1);
        if (rem > halfway || (rem == halfway && (q & 1u)))
            ++q;
        return (uint16_t)(sign | q);
    }
    uint32_t h = ((absx >> 13) - (112u << 10));
    const uint32_t rem = absx & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u)))
        ++h;
    return (uint16_t)(sign | h);
}

static float prev_corr(float c, float beta) {
    return beta > 0.f ? fmaxf((c - (1.f - beta)) / beta, 0.f) : 0.f;
}

static float to_norm(float m, float v, float c1, float c2, float eps) {
    if (c1 <= 0.f || c2 <= 0.f)
        return 0.f;
    return (m / c1) / (sqrtf(fmaxf(v, 0.f) / c2) + eps);
}

static float log_to_second(float ls) {
    const float s = 1e-15f * expm1f(ls);
    return s * s;
}

void orc_sh_adam_rows(int rows, int stride, int active, float* param, const float* grad,
                      uint16_t* first, uint8_t* packed, float* bounds, float lr, float rest_lr,
                      float b1, float b2, float c1, float c2, float eps, float reg) {
    if (stride > 64)
        return; /* rows hold at most 16 RGB bases (48 columns) */
    for (int r = 0; r < rows; ++r) {
        float* p = param + (size_t)r * stride;
        const float* gr = grad + (size_t)r * stride;
        uint16_t* f = first + (size_t)r * stride;
        uint8_t* pk = packed + (size_t)r * stride;
        float* bd = bounds + 4 * (size_t)r;
        float b[4] = {bd[0], bd[1], bd[2], bd[3]};
        if (!isfinite(b[0]) || !isfinite(b[1])) b[0] = b[1] = 0.f;
        if (!isfinite(b[2]) || !isfinite(b[3])) b[2] = b[3] = 0.f;
        float ls[64];
        float dmin = 1e30f, dmax = -1e30f, rmin = 1e30f, rmax = -1e30f;
        for (int col = 0; col < stride; ++col) {
            const int dc = col < 3;
            const float lo = dc ? b[0] : b[2], hi = dc ? b[1] : b[3];
            float l = lo + (hi - lo) * ((float)pk[col] * (1.f / 255.f));
            const float g2 = log_to_second(l);
            const float stored = half_to_float(f[col]);
            const float pc1 = prev_corr(c1, b1), pc2 = prev_corr(c2, b2);
            float g1 = 0.f;
            if (pc1 > 0.f) {
                const float sv = pc2 > 0.f ? sqrtf(fmaxf(g2, 0.f) / pc2) : 0.f;
                g1 = stored * (sv + eps) * pc1;
            }
            if (col >= active) {
                if (!isfinite(g1)) g1 = 0.f;
                if (!isfinite(l)) { l = 0.f; g1 = 0.f; }
                const float enc = to_norm(g1, log_to_second(l), c1, c2, eps);
                f[col] = float_to_half(isfinite(enc) ? enc : 0.f);
            } else {
                float gg = gr[col];
                const float prev = p[col];
                if (reg > 0.f && col >= 3 && isfinite(prev)) gg += reg * prev;
                if (!isfinite(prev) || !isfinite(gg)) {
                    f[col] = 0;
                    p[col] = isfinite(prev) ? prev : 0.f;
                    l = 0.f;
                } else {
                    const float m = b1 * g1 + (1.f - b1) * gg;
                    const float v = b2 * g2 + (1.f - b2) * gg * gg;
                    if (!isfinite(m) || !isfinite(v)) {
                        f[col] = 0;
                        l = 0.f;
                    } else {
                        const float nrm = to_norm(m, v, c1, c2, eps);
                        const float cand = prev - (col >= 3 ? rest_lr : lr) * nrm;
                        p[col] = isfinite(cand) ? cand : prev;
                        f[col] = float_to_half(nrm);
                        l = log1pf(sqrtf(fmaxf(v, 0.f)) * (1.f / 1e-15f));
                        if (!isfinite(l)) l = 0.f;
                    }
                }
            }
            ls[col] = l;
            if (dc) { dmin = fminf(dmin, l); dmax = fmaxf(dmax, l); }
            else { rmin = fminf(rmin, l); rmax = fmaxf(rmax, l); }
        }
        if (stride <= 3) rmin = rmax = 0.f;
        bd[0] = dmin; bd[1] = dmax; bd[2] = rmin; bd[3] = rmax;
        for (int col = 0; col < stride; ++col) {
            const float lo = col < 3 ? dmin : rmin, hi = col < 3 ? dmax : rmax;
            const float range = fmaxf(hi - lo, 1e-15f);
            const float code = fminf(fmaxf(roundf(255.f * (ls[col] - lo) / range), 0.f), 255.f);
            pk[col] = (uint8_t)code;
        }
    }
}
