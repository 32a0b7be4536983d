/*
 * gsn_oracle.c - CPU oracle of the 3DGS training hot path (see gsn_oracle.h).
 *
 * TEST INFRASTRUCTURE ONLY: a restatement of the reference's algorithm in plain
 * C, FP64 wherever the reference computes a real-valued quantity and exact
 * integer arithmetic for the record ordering. Each function names the
 * reference lines it follows. Compiled with -ffp-contract=off so that no fused
 * multiply-add changes the FP64 results between builds.
 */
#include "gsn_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_TILE 16
#define ORC_LOW_PASS 0.3
#define ORC_FOV_CLAMP 1.3

static const double kC0 = 0.28209479177387814;
static const double kC1 = 0.4886025119029199;
static const double kC2a = 1.0925484305920792;
static const double kC2b = 0.31539156525252005;
static const double kC2c = 0.5462742152960396;
static const double kC3a = 0.5900435899266435;
static const double kC3b = 2.890611442640554;
static const double kC3c = 0.4570457994644658;
static const double kC3d = 0.3731763325901154;
static const double kC3e = 1.445305721320277;

int orc_set_threads(int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
    return omp_get_max_threads();
#else
    (void)threads;
    return 1;
#endif
}

void orc_free(void* ptr) { free(ptr); }

static double clampd(double x, double lo, double hi) { return x < lo ? lo : (x > hi ? hi : x); }

/* Real SH basis up to degree 3 (cpu_reference.h:11-21; renderer.cu:68-106). */
static void sh_basis(double x, double y, double z, double b[16]) {
    b[0] = kC0;
    b[1] = -kC1 * y;
    b[2] = kC1 * z;
    b[3] = -kC1 * x;
    b[4] = kC2a * x * y;
    b[5] = -kC2a * y * z;
    b[6] = kC2b * (2 * z * z - x * x - y * y);
    b[7] = -kC2a * x * z;
    b[8] = kC2c * (x * x - y * y);
    b[9] = -kC3a * y * (3 * x * x - y * y);
    b[10] = kC3b * x * y * z;
    b[11] = -kC3c * y * (4 * z * z - x * x - y * y);
    b[12] = kC3d * z * (2 * z * z - 3 * x * x - 3 * y * y);
    b[13] = -kC3c * x * (4 * z * z - x * x - y * y);
    b[14] = kC3e * z * (x * x - y * y);
    b[15] = -kC3a * x * (x * x - 3 * y * y);
}

/* Gradient of every basis polynomial w.r.t. its (x, y, z) arguments, g[k][axis]
 * (the closed forms of solver.cu:245-302). */
static void sh_basis_gradient(double x, double y, double z, double g[16][3]) {
    memset(g, 0, sizeof(double) * 48);
    g[1][1] = -kC1;
    g[2][2] = kC1;
    g[3][0] = -kC1;
    g[4][0] = kC2a * y; g[4][1] = kC2a * x;
    g[5][1] = -kC2a * z; g[5][2] = -kC2a * y;
    g[6][0] = -2 * kC2b * x; g[6][1] = -2 * kC2b * y; g[6][2] = 4 * kC2b * z;
    g[7][0] = -kC2a * z; g[7][2] = -kC2a * x;
    g[8][0] = 2 * kC2c * x; g[8][1] = -2 * kC2c * y;
    g[9][0] = -6 * kC3a * x * y; g[9][1] = -3 * kC3a * (x * x - y * y);
    g[10][0] = kC3b * y * z; g[10][1] = kC3b * x * z; g[10][2] = kC3b * x * y;
    g[11][0] = 2 * kC3c * x * y; g[11][1] = -kC3c * (4 * z * z - x * x - 3 * y * y); g[11][2] = -8 * kC3c * y * z;
    g[12][0] = -6 * kC3d * x * z; g[12][1] = -6 * kC3d * y * z; g[12][2] = kC3d * (6 * z * z - 3 * x * x - 3 * y * y);
    g[13][0] = -kC3c * (4 * z * z - 3 * x * x - y * y); g[13][1] = 2 * kC3c * x * y; g[13][2] = -8 * kC3c * x * z;
    g[14][0] = 2 * kC3e * x * z; g[14][1] = -2 * kC3e * y * z; g[14][2] = kC3e * (x * x - y * y);
    g[15][0] = -3 * kC3a * (x * x - y * y); g[15][1] = 6 * kC3a * x * y;
}

/* Axis-angle -> rotation matrix, identity below 1e-8 (renderer.cu:35-66). */
static void rotation_matrix(double wx, double wy, double wz, double R[9]) {
    double angle = sqrt(wx * wx + wy * wy + wz * wz);
    if (angle < 1e-8) {
        memset(R, 0, 9 * sizeof(double));
        R[0] = R[4] = R[8] = 1.0;
        return;
    }
    double x = wx / angle, y = wy / angle, z = wz / angle;
    double c = cos(angle), s = sin(angle), t = 1.0 - c;
    R[0] = c + t * x * x; R[1] = t * x * y - s * z; R[2] = t * x * z + s * y;
    R[3] = t * x * y + s * z; R[4] = c + t * y * y; R[5] = t * y * z - s * x;
    R[6] = t * x * z - s * y; R[7] = t * y * z + s * x; R[8] = c + t * z * z;
}

static void camera_center(const gsn_camera* cam, double C[3]) {
    for (int a = 0; a < 3; ++a) {
        C[a] = 0;
        for (int r = 0; r < 3; ++r) C[a] -= (double)cam->R_c_w[r * 3 + a] * cam->t_c_w[r];
    }
}

/* renderer.cu:108-221 (FP64, as cpu_reference.h:45-85 evaluates it). */
void orc_project(const float* params, int n, const gsn_camera* cam, int sh_degree, orc_proj* out) {
    if (sh_degree < 0) sh_degree = 0;
    if (sh_degree > 3) sh_degree = 3;
    const int64_t N = n;
    const int K = (sh_degree + 1) * (sh_degree + 1);
    double C[3];
    camera_center(cam, C);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        orc_proj* o = out + i;
        memset(o, 0, sizeof(*o));
        double pos[3] = {params[0 * N + i], params[1 * N + i], params[2 * N + i]};
        double pc[3];
        for (int r = 0; r < 3; ++r)
            pc[r] = (double)cam->R_c_w[r * 3] * pos[0] + (double)cam->R_c_w[r * 3 + 1] * pos[1] +
                    (double)cam->R_c_w[r * 3 + 2] * pos[2] + cam->t_c_w[r];
        double z = pc[2];
        double near = fmax(cam->near_depth, 1e-6);
        if (z <= near || z > fmax(cam->far_depth, near)) continue;
        double Rg[9];
        rotation_matrix(params[6 * N + i], params[7 * N + i], params[8 * N + i], Rg);
        double s[3] = {exp(params[3 * N + i]), exp(params[4 * N + i]), exp(params[5 * N + i])};
        double M[9], V[9];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c)
                M[r * 3 + c] = ((double)cam->R_c_w[r * 3] * Rg[c] + (double)cam->R_c_w[r * 3 + 1] * Rg[3 + c] +
                                (double)cam->R_c_w[r * 3 + 2] * Rg[6 + c]) * s[c];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c)
                V[r * 3 + c] = M[r * 3] * M[c * 3] + M[r * 3 + 1] * M[c * 3 + 1] + M[r * 3 + 2] * M[c * 3 + 2];
        double lim_x = ORC_FOV_CLAMP * 0.5 * cam->width / cam->fx;
        double lim_y = ORC_FOV_CLAMP * 0.5 * cam->height / cam->fy;
        double x = clampd(pc[0] / z, -lim_x, lim_x) * z;
        double y = clampd(pc[1] / z, -lim_y, lim_y) * z;
        double J[6] = {cam->fx / z, 0, -cam->fx * x / (z * z), 0, cam->fy / z, -cam->fy * y / (z * z)};
        double JV[6];
        for (int r = 0; r < 2; ++r)
            for (int c = 0; c < 3; ++c) JV[r * 3 + c] = J[r * 3] * V[c] + J[r * 3 + 1] * V[3 + c] + J[r * 3 + 2] * V[6 + c];
        double a = JV[0] * J[0] + JV[1] * J[1] + JV[2] * J[2] + ORC_LOW_PASS;
        double b = JV[0] * J[3] + JV[1] * J[4] + JV[2] * J[5];
        double c = JV[3] * J[3] + JV[4] * J[4] + JV[5] * J[5] + ORC_LOW_PASS;
        double det = a * c - b * b;
        if (!(det > 0)) continue;
        double mid = 0.5 * (a + c);
        double radius = ceil(3.0 * sqrt(mid + sqrt(fmax(0.1, mid * mid - det))));
        double u = cam->fx * pc[0] / z + cam->cx;
        double v = cam->fy * pc[1] / z + cam->cy;
        if (!isfinite(radius) || !isfinite(u) || !isfinite(v)) continue;
        int rx0 = (int)clampd((u - radius) / ORC_TILE, 0.0, cam->tile_count_x);
        int ry0 = (int)clampd((v - radius) / ORC_TILE, 0.0, cam->tile_count_y);
        int rx1 = (int)clampd((u + radius + ORC_TILE - 1) / ORC_TILE, 0.0, cam->tile_count_x);
        int ry1 = (int)clampd((v + radius + ORC_TILE - 1) / ORC_TILE, 0.0, cam->tile_count_y);
        if (rx0 >= rx1 || ry0 >= ry1) continue;
        o->visible = 1;
        o->rect[0] = rx0; o->rect[1] = ry0; o->rect[2] = rx1; o->rect[3] = ry1;
        o->depth = z;
        o->u = u; o->v = v;
        o->cov[0] = a; o->cov[1] = b; o->cov[2] = c;
        o->conic[0] = c / det; o->conic[1] = -b / det; o->conic[2] = a / det;
        o->opacity = 1.0 / (1.0 + exp(-(double)params[9 * N + i]));
        o->radius = radius;
        double d[3] = {pos[0] - C[0], pos[1] - C[1], pos[2] - C[2]};
        double len = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        double basis[16];
        sh_basis(d[0] / len, d[1] / len, d[2] / len, basis);
        for (int ch = 0; ch < 3; ++ch) {
            double value = 0;
            for (int k = 0; k < K; ++k) value += basis[k] * params[(GSN_SH_INDEX + ch * 16 + k) * N + i];
            o->rgb_raw[ch] = value + 0.5;
            o->rgb[ch] = fmax(value + 0.5, 0.0);
        }
    }
}

/* ------------------------------------------------------------ record order */
typedef struct { uint64_t key; int32_t id; } orc_rec;

static void merge_sort_records(orc_rec* a, orc_rec* tmp, int64_t n) {
    for (int64_t width = 1; width < n; width *= 2) {
        for (int64_t lo = 0; lo < n; lo += 2 * width) {
            int64_t mid = lo + width < n ? lo + width : n;
            int64_t hi = lo + 2 * width < n ? lo + 2 * width : n;
            int64_t i = lo, j = mid, k = lo;
            while (i < mid && j < hi) tmp[k++] = (a[j].key < a[i].key) ? a[j++] : a[i++];
            while (i < mid) tmp[k++] = a[i++];
            while (j < hi) tmp[k++] = a[j++];
        }
        memcpy(a, tmp, (size_t)n * sizeof(orc_rec));
    }
}

/* renderer.cu:223-271 (record write in id order, rect row-major), 541-563
 * (stable sort of the 64-bit keys) and IdentifyTileOffsetsKernel. */
int64_t orc_sort_records(const uint32_t* depth_bits, const int* rects, const int* counts, int n,
                         int tile_count_x, int tile_count_y, int32_t* out_ids, int64_t* out_offsets) {
    int64_t total = 0;
    for (int i = 0; i < n; ++i) total += counts[i];
    int64_t tiles = (int64_t)tile_count_x * tile_count_y;
    orc_rec* recs = (orc_rec*)malloc((size_t)(total > 0 ? total : 1) * sizeof(orc_rec));
    orc_rec* tmp = (orc_rec*)malloc((size_t)(total > 0 ? total : 1) * sizeof(orc_rec));
    int64_t w = 0;
    for (int i = 0; i < n; ++i) {
        if (counts[i] <= 0) continue;
        const int* r = rects + 4 * i;
        int width = r[2] - r[0];
        for (int k = 0; k < counts[i]; ++k) {
            uint64_t tile = (uint64_t)(r[1] + k / width) * tile_count_x + r[0] + k % width;
            recs[w].key = (tile << 32) | depth_bits[i];
            recs[w].id = i;
            ++w;
        }
    }
    merge_sort_records(recs, tmp, total);
    for (int64_t t = 0; t <= tiles; ++t) out_offsets[t] = 0;
    for (int64_t r = 0; r < total; ++r) {
        out_ids[r] = recs[r].id;
        int tile = (int)(recs[r].key >> 32);
        int prev = r == 0 ? -1 : (int)(recs[r - 1].key >> 32);
        for (int e = prev + 1; e <= tile; ++e) out_offsets[e] = r;
        if (r == total - 1)
            for (int64_t e = tile + 1; e <= tiles; ++e) out_offsets[e] = total;
    }
    free(recs);
    free(tmp);
    return total;
}

/* ------------------------------------------------------------ tile lists */
static const orc_proj* g_sort_proj;
static int cmp_depth(const void* pa, const void* pb) {
    int a = *(const int*)pa, b = *(const int*)pb;
    double da = g_sort_proj[a].depth, db = g_sort_proj[b].depth;
    if (da < db) return -1;
    if (da > db) return 1;
    return a < b ? -1 : (a > b);
}

/* Stable (depth, id) order of cpu_reference.h:36-41 split into per-tile lists. */
void orc_tile_lists(const orc_proj* p, int n, const gsn_camera* cam, int64_t** offsets_out, int32_t** ids_out) {
    int64_t tiles = (int64_t)cam->tile_count_x * cam->tile_count_y;
    int* order = (int*)malloc((size_t)(n > 0 ? n : 1) * sizeof(int));
    int m = 0;
    for (int i = 0; i < n; ++i)
        if (p[i].visible) order[m++] = i;
    g_sort_proj = p;
    qsort(order, (size_t)m, sizeof(int), cmp_depth);
    int64_t* offsets = (int64_t*)calloc((size_t)tiles + 1, sizeof(int64_t));
    for (int k = 0; k < m; ++k) {
        const int* r = p[order[k]].rect;
        for (int ty = r[1]; ty < r[3]; ++ty)
            for (int tx = r[0]; tx < r[2]; ++tx) offsets[(int64_t)ty * cam->tile_count_x + tx + 1]++;
    }
    for (int64_t t = 0; t < tiles; ++t) offsets[t + 1] += offsets[t];
    int64_t total = offsets[tiles];
    int32_t* ids = (int32_t*)malloc((size_t)(total > 0 ? total : 1) * sizeof(int32_t));
    int64_t* fill = (int64_t*)malloc((size_t)(tiles > 0 ? tiles : 1) * sizeof(int64_t));
    memcpy(fill, offsets, (size_t)tiles * sizeof(int64_t));
    for (int k = 0; k < m; ++k) {
        const int* r = p[order[k]].rect;
        for (int ty = r[1]; ty < r[3]; ++ty)
            for (int tx = r[0]; tx < r[2]; ++tx) ids[fill[(int64_t)ty * cam->tile_count_x + tx]++] = order[k];
    }
    free(fill);
    free(order);
    *offsets_out = offsets;
    *ids_out = ids;
}

/* ------------------------------------------------------------ blending */
typedef struct {
    double power, raw_alpha, alpha;
    int skip;
} orc_pair;

/* One (pixel, Gaussian) evaluation with the thresholds of renderer.cu:311-323. */
static orc_pair eval_pair(const orc_proj* g, double px, double py) {
    orc_pair e;
    double dx = g->u - px, dy = g->v - py;
    e.power = -0.5 * (g->conic[0] * dx * dx + g->conic[2] * dy * dy) - g->conic[1] * dx * dy;
    e.raw_alpha = g->opacity * exp(e.power);
    e.alpha = e.raw_alpha < 0.99 ? e.raw_alpha : 0.99;
    e.skip = e.power > 0 || e.alpha < 1.0 / 255.0;
    return e;
}

static void tile_range(const gsn_camera* cam, int* tb, int* te) {
    int tiles = cam->tile_count_x * cam->tile_count_y;
    if (*te <= 0 || *te > tiles) *te = tiles;
    if (*tb < 0) *tb = 0;
}

void orc_render(const orc_proj* p, const gsn_camera* cam, const int64_t* offsets, const int32_t* ids,
                const double* background, double* image, double* final_t, int* contributors, int tile_begin,
                int tile_end) {
    tile_range(cam, &tile_begin, &tile_end);
#pragma omp parallel for schedule(dynamic, 4)
    for (int tile = tile_begin; tile < tile_end; ++tile) {
        int tx = tile % cam->tile_count_x, ty = tile / cam->tile_count_x;
        for (int ly = 0; ly < ORC_TILE; ++ly)
            for (int lx = 0; lx < ORC_TILE; ++lx) {
                int x = tx * ORC_TILE + lx, y = ty * ORC_TILE + ly;
                if (x >= cam->width || y >= cam->height) continue;
                double T = 1.0, col[3] = {0, 0, 0};
                int consumed = 0;
                for (int64_t r = offsets[tile]; r < offsets[tile + 1]; ++r) {
                    const orc_proj* g = p + ids[r];
                    orc_pair e = eval_pair(g, x, y);
                    if (e.skip) continue;
                    double nextT = T * (1 - e.alpha);
                    if (nextT < 1e-4) break;
                    for (int c = 0; c < 3; ++c) col[c] += g->rgb[c] * e.alpha * T;
                    T = nextT;
                    consumed = (int)(r - offsets[tile]) + 1;
                }
                int64_t pix = (int64_t)y * cam->width + x;
                for (int c = 0; c < 3; ++c) image[pix * 3 + c] = col[c] + T * background[c];
                if (final_t) final_t[pix] = T;
                if (contributors) contributors[pix] = consumed;
            }
    }
}

/* ------------------------------------------------------------ loss */
static void gaussian_window(double w[11]) {
    double sum = 0;
    for (int i = 0; i < 11; ++i) {
        double d = i - 5;
        w[i] = exp(-d * d / (2 * 1.5 * 1.5));
        sum += w[i];
    }
    for (int i = 0; i < 11; ++i) w[i] /= sum;
}

/* Separable zero-padded 11-tap filter of a single-channel band [y0, y1) x [0, W)
 * of an H-row image; rows outside [0, H) are zero. src and dst hold (y1 - y0) rows. */
static void filter_band(const double* src, double* dst, double* tmp, int width, int height, int y0, int y1,
                        const double w[11]) {
    int rows = y1 - y0;
    for (int r = 0; r < rows; ++r)
        for (int x = 0; x < width; ++x) {
            double s = 0;
            for (int k = 0; k < 11; ++k) {
                int xx = x + k - 5;
                if (xx >= 0 && xx < width) s += w[k] * src[(int64_t)r * width + xx];
            }
            tmp[(int64_t)r * width + x] = s;
        }
    for (int r = 0; r < rows; ++r)
        for (int x = 0; x < width; ++x) {
            double s = 0;
            for (int k = 0; k < 11; ++k) {
                int rr = r + k - 5;
                int yy = y0 + rr;
                if (yy >= 0 && yy < height && rr >= 0 && rr < rows) s += w[k] * tmp[(int64_t)rr * width + x];
            }
            dst[(int64_t)r * width + x] = s;
        }
}

/* cpu_reference.h:120-152. */
double orc_loss(const double* image, const uint8_t* target, int width, int height) {
    double w[11];
    gaussian_window(w);
    int64_t P = (int64_t)width * height;
    double* buf = (double*)malloc(sizeof(double) * P * 8);
    double *a = buf, *b = buf + P, *tmp = buf + 7 * P;
    double l1 = 0, ssim = 0;
    double* f = (double*)malloc(sizeof(double) * P * 5);
    for (int c = 0; c < 3; ++c) {
        for (int64_t i = 0; i < P; ++i) {
            a[i] = image[i * 3 + c];
            b[i] = target[i * 3 + c] / 255.0;
            l1 += fabs(a[i] - b[i]);
        }
        double* prod = buf + 2 * P;
        double* src[5] = {a, b, NULL, NULL, NULL};
        for (int k = 0; k < 5; ++k) {
            if (k >= 2) {
                for (int64_t i = 0; i < P; ++i)
                    prod[i] = k == 2 ? a[i] * a[i] : (k == 3 ? b[i] * b[i] : a[i] * b[i]);
                src[k] = prod;
            }
            filter_band(src[k], f + k * P, tmp, width, height, 0, height, w);
        }
        for (int64_t i = 0; i < P; ++i) {
            double ma = f[i], mb = f[P + i];
            double va = f[2 * P + i] - ma * ma, vb = f[3 * P + i] - mb * mb, cov = f[4 * P + i] - ma * mb;
            ssim += (2 * ma * mb + 0.0001) * (2 * cov + 0.0009) / ((ma * ma + mb * mb + 0.0001) * (va + vb + 0.0009));
        }
    }
    free(f);
    free(buf);
    double count = 3.0 * (double)P;
    return 0.8 * l1 / count + 0.2 * (1 - ssim / count);
}

/* Evaluation metrics of held-out views, as the reference documents them
 * (README.md "Metrics are averaged over the held-out views..."): RGB clamped to
 * [0, 1], PSNR of the RGB mean squared error, SSIM with the 11 x 11 Gaussian
 * window (sigma 1.5) and the loss's zero padding and constants, mean L1.
 * out[0..3] = PSNR (dB), mean SSIM, mean L1, MSE. FP64 throughout. */
void orc_eval_metrics(const double* image, const uint8_t* target, int width, int height, double* out) {
    double w[11];
    gaussian_window(w);
    int64_t P = (int64_t)width * height;
    double* buf = (double*)malloc(sizeof(double) * P * 4);
    double* f = (double*)malloc(sizeof(double) * P * 5);
    double *a = buf, *b = buf + P, *prod = buf + 2 * P, *tmp = buf + 3 * P;
    double l1 = 0, sq = 0, ssim = 0;
    for (int c = 0; c < 3; ++c) {
        for (int64_t i = 0; i < P; ++i) {
            double v = image[i * 3 + c];
            a[i] = v < 0 ? 0 : (v > 1 ? 1 : v);
            b[i] = target[i * 3 + c] / 255.0;
            l1 += fabs(a[i] - b[i]);
            sq += (a[i] - b[i]) * (a[i] - b[i]);
        }
        double* src[5] = {a, b, NULL, NULL, NULL};
        for (int k = 0; k < 5; ++k) {
            if (k >= 2) {
                for (int64_t i = 0; i < P; ++i)
                    prod[i] = k == 2 ? a[i] * a[i] : (k == 3 ? b[i] * b[i] : a[i] * b[i]);
                src[k] = prod;
            }
            filter_band(src[k], f + k * P, tmp, width, height, 0, height, w);
        }
        for (int64_t i = 0; i < P; ++i) {
            double ma = f[i], mb = f[P + i];
            double va = f[2 * P + i] - ma * ma, vb = f[3 * P + i] - mb * mb, cov = f[4 * P + i] - ma * mb;
            ssim += (2 * ma * mb + 0.0001) * (2 * cov + 0.0009) / ((ma * ma + mb * mb + 0.0001) * (va + vb + 0.0009));
        }
    }
    free(f);
    free(buf);
    double count = 3.0 * (double)P;
    double mse = sq / count;
    out[0] = mse > 0 ? -10.0 * log10(mse) : INFINITY;
    out[1] = ssim / count;
    out[2] = l1 / count;
    out[3] = mse;
}

/* Analytic gradient of orc_loss: L1 sign term plus the SSIM chain through the
 * two separable filter passes, the quantity solver.cu:26-168 evaluates in FP32.
 * Output rows [row_begin, row_end) (all rows when row_end <= 0). */
void orc_loss_gradient(const double* image, const uint8_t* target, int width, int height, double* gradient,
                       int row_begin, int row_end) {
    if (row_end <= 0 || row_end > height) row_end = height;
    if (row_begin < 0) row_begin = 0;
    double w[11];
    gaussian_window(w);
    const double norm = 1.0 / (3.0 * (double)width * height);
    /* band of centres whose SSIM terms reach the output rows, and the image rows
     * their moments need */
    int cy0 = row_begin - 5 < 0 ? 0 : row_begin - 5, cy1 = row_end + 5 > height ? height : row_end + 5;
    int iy0 = cy0 - 5 < 0 ? 0 : cy0 - 5, iy1 = cy1 + 5 > height ? height : cy1 + 5;
    int irows = iy1 - iy0;
    int64_t IP = (int64_t)irows * width;
#pragma omp parallel for schedule(static)
    for (int c = 0; c < 3; ++c) {
        double* buf = (double*)malloc(sizeof(double) * IP * 12);
        double *a = buf, *b = buf + IP, *prod = buf + 2 * IP, *tmp = buf + 3 * IP, *f = buf + 4 * IP;
        double *ga = buf + 9 * IP, *gb = buf + 10 * IP, *gc = buf + 11 * IP;
        for (int64_t i = 0; i < IP; ++i) {
            int64_t src = (int64_t)iy0 * width + i;
            a[i] = image[src * 3 + c];
            b[i] = target[src * 3 + c] / 255.0;
        }
        double* srcs[5] = {a, b, prod, prod, prod};
        for (int k = 0; k < 5; ++k) {
            if (k >= 2)
                for (int64_t i = 0; i < IP; ++i) prod[i] = k == 2 ? a[i] * a[i] : (k == 3 ? b[i] * b[i] : a[i] * b[i]);
            filter_band(srcs[k], f + k * IP, tmp, width, height, iy0, iy1, w);
        }
        /* per-centre partials (solver.cu:105-128): a = dSSIM/dmu_x, b = dSSIM/dE[xy], c = dSSIM/dE[x^2] */
        for (int64_t i = 0; i < IP; ++i) {
            int y = iy0 + (int)(i / width);
            double A = 0, B = 0, Cc = 0;
            if (y >= cy0 && y < cy1) {
                double m = f[i], nn = f[IP + i];
                double D = m * m + nn * nn + 0.0001;
                double E = f[2 * IP + i] - m * m + f[3 * IP + i] - nn * nn + 0.0009;
                double lum = (2 * m * nn + 0.0001) / D;
                double cs = (2 * (f[4 * IP + i] - m * nn) + 0.0009) / E;
                B = 2 * lum / E;
                Cc = -lum * cs / E;
                A = 2 * (nn - m * lum) / D * cs - nn * B - 2 * m * Cc;
            }
            ga[i] = A; gb[i] = B; gc[i] = Cc;
        }
        double* fa = f;               /* reuse moment storage */
        double* fb = f + IP;
        double* fc = f + 2 * IP;
        filter_band(ga, fa, tmp, width, height, iy0, iy1, w);
        filter_band(gb, fb, tmp, width, height, iy0, iy1, w);
        filter_band(gc, fc, tmp, width, height, iy0, iy1, w);
        for (int y = row_begin; y < row_end; ++y)
            for (int x = 0; x < width; ++x) {
                int64_t li = (int64_t)(y - iy0) * width + x;
                int64_t gi = ((int64_t)y * width + x) * 3 + c;
                double I = a[li], Tt = b[li];
                double r = I - Tt;
                double l1 = (double)(r > 0) - (double)(r < 0);
                double ssim = -(fa[li] + Tt * fb[li] + 2 * I * fc[li]);
                gradient[gi] = (0.8 * l1 + 0.2 * ssim) * norm;
            }
        free(buf);
    }
}

/* ------------------------------------------------------------ backward */
/* solver.cu:325-466: front-to-back replay of each pixel against its final
 * colour, per-pixel contributions summed per Gaussian. */
void orc_backward(const orc_proj* p, int n, const gsn_camera* cam, const int64_t* offsets, const int32_t* ids,
                  const double* image, const double* image_gradient, double* grad9, double* abs2, int tile_begin,
                  int tile_end) {
    const int64_t N = n;
    tile_range(cam, &tile_begin, &tile_end);
#pragma omp parallel for schedule(dynamic, 4)
    for (int tile = tile_begin; tile < tile_end; ++tile) {
        int tx = tile % cam->tile_count_x, ty = tile / cam->tile_count_x;
        for (int ly = 0; ly < ORC_TILE; ++ly)
            for (int lx = 0; lx < ORC_TILE; ++lx) {
                int x = tx * ORC_TILE + lx, y = ty * ORC_TILE + ly;
                if (x >= cam->width || y >= cam->height) continue;
                int64_t pix = (int64_t)y * cam->width + x;
                const double* fin = image + pix * 3;
                const double* gI = image_gradient + pix * 3;
                double T = 1.0, prefix[3] = {0, 0, 0};
                for (int64_t r = offsets[tile]; r < offsets[tile + 1]; ++r) {
                    int id = ids[r];
                    const orc_proj* g = p + id;
                    orc_pair e = eval_pair(g, x, y);
                    if (e.skip) continue;
                    double nextT = T * (1 - e.alpha);
                    if (nextT < 1e-4) break;
                    double weight = e.alpha * T, dalpha = 0, contrib[9] = {0};
                    for (int c = 0; c < 3; ++c) {
                        dalpha += gI[c] * (prefix[c] + T * g->rgb[c] - fin[c]) / (1 - e.alpha);
                        contrib[6 + c] = weight * gI[c];
                    }
                    if (e.raw_alpha < 0.99) {
                        double common = dalpha * e.raw_alpha;
                        double dx = g->u - x, dy = g->v - y;
                        double qx = g->conic[0] * dx + g->conic[1] * dy;
                        double qy = g->conic[1] * dx + g->conic[2] * dy;
                        contrib[0] = -common * qx;
                        contrib[1] = -common * qy;
                        contrib[2] = 0.5 * common * qx * qx;
                        contrib[3] = common * qx * qy;
                        contrib[4] = 0.5 * common * qy * qy;
                        contrib[5] = common * (1 - g->opacity);
                    }
                    for (int c = 0; c < 3; ++c) prefix[c] += g->rgb[c] * weight;
                    T = nextT;
                    for (int f = 0; f < 9; ++f) {
                        if (contrib[f] == 0) continue;
#pragma omp atomic
                        grad9[f * N + id] += contrib[f];
                    }
                    double a0 = fabs(contrib[0]), a1 = fabs(contrib[1]);
#pragma omp atomic
                    abs2[id] += a0;
#pragma omp atomic
                    abs2[N + id] += a1;
                }
            }
    }
}

void orc_projection_statistics(const orc_proj* p, int n, const gsn_camera* cam, const double* grad9,
                               const double* abs2, double* stats, double* abs_stats) {
    for (int i = 0; i < n; ++i) {
        double x = grad9[i] * (0.5 * cam->width), y = grad9[(int64_t)n + i] * (0.5 * cam->height);
        double ax = abs2[i] * (0.5 * cam->width), ay = abs2[(int64_t)n + i] * (0.5 * cam->height);
        stats[i] = sqrt(x * x + y * y);
        stats[(int64_t)n + i] = p[i].visible ? 1.0 : 0.0;
        abs_stats[i] = sqrt(ax * ax + ay * ay);
    }
}

/* ------------------------------------------------------------ chain rule */
/* solver.cu:492-623 in FP64: 2D mean / covariance / colour gradients to
 * position, log-scale, axis-angle (right Jacobian), opacity logit and SH. */
void orc_map_gradients(const float* params, int n, const gsn_camera* cam, int sh_degree, const double* grad9,
                       double* grad58) {
    if (sh_degree < 0) sh_degree = 0;
    if (sh_degree > 3) sh_degree = 3;
    const int64_t N = n;
    const int K = (sh_degree + 1) * (sh_degree + 1);
    double Cc[3];
    camera_center(cam, Cc);
    double Rc[9];
    for (int k = 0; k < 9; ++k) Rc[k] = cam->R_c_w[k];
#pragma omp parallel for schedule(static)
    for (int id = 0; id < n; ++id) {
        double in[9];
        int active = 0;
        for (int j = 0; j < 9; ++j) {
            in[j] = grad9[j * N + id];
            active |= in[j] != 0.0;
        }
        for (int r = 0; r < 58; ++r) grad58[r * N + id] = 0;
        if (!active) continue;
        double pos[3] = {params[id], params[N + id], params[2 * N + id]};
        double w[3] = {params[6 * N + id], params[7 * N + id], params[8 * N + id]};
        double Rg[9], CR[9], s2[3], V[9], pc[3];
        rotation_matrix(w[0], w[1], w[2], Rg);
        for (int r = 0; r < 3; ++r) {
            pc[r] = cam->t_c_w[r];
            for (int c = 0; c < 3; ++c) {
                pc[r] += Rc[r * 3 + c] * pos[c];
                CR[r * 3 + c] = Rc[r * 3] * Rg[c] + Rc[r * 3 + 1] * Rg[3 + c] + Rc[r * 3 + 2] * Rg[6 + c];
            }
            double s = exp(params[(3 + r) * N + id]);
            s2[r] = s * s;
        }
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                V[r * 3 + c] = 0;
                for (int j = 0; j < 3; ++j) V[r * 3 + c] += CR[r * 3 + j] * s2[j] * CR[c * 3 + j];
            }
        double iz = 1.0 / pc[2];
        double nx = pc[0] * iz, ny = pc[1] * iz;
        double lx = ORC_FOV_CLAMP * 0.5 * cam->width / cam->fx, ly = ORC_FOV_CLAMP * 0.5 * cam->height / cam->fy;
        double jx = clampd(nx, -lx, lx), jy = clampd(ny, -ly, ly);
        double P[6] = {cam->fx * iz, 0, -cam->fx * jx * iz, 0, cam->fy * iz, -cam->fy * jy * iz};
        double PV[6] = {0}, LP[6] = {0};
        for (int r = 0; r < 2; ++r)
            for (int c = 0; c < 3; ++c)
                for (int j = 0; j < 3; ++j) {
                    PV[r * 3 + c] += P[r * 3 + j] * V[j * 3 + c];
                    LP[r * 3 + c] += P[r * 3 + j] * CR[j * 3 + c];
                }
        /* colour and its view-direction derivative */
        double d[3] = {pos[0] - Cc[0], pos[1] - Cc[1], pos[2] - Cc[2]};
        double il = 1.0 / sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        double ux = d[0] * il, uy = d[1] * il, uz = d[2] * il;
        double basis[16], bg[16][3];
        sh_basis(ux, uy, uz, basis);
        sh_basis_gradient(ux, uy, uz, bg);
        double color[3], dcol[3][3];
        for (int ch = 0; ch < 3; ++ch) {
            double value = 0, der[3] = {0, 0, 0};
            for (int k = 0; k < K; ++k) {
                double coef = params[(GSN_SH_INDEX + ch * 16 + k) * N + id];
                value += coef * basis[k];
                for (int a = 0; a < 3; ++a) der[a] += coef * bg[k][a];
            }
            color[ch] = value + 0.5;
            double radial = der[0] * ux + der[1] * uy + der[2] * uz;
            dcol[ch][0] = (der[0] - radial * ux) * il;
            dcol[ch][1] = (der[1] - radial * uy) * il;
            dcol[ch][2] = (der[2] - radial * uz) * il;
        }
        double right[3];
        for (int axis = 0; axis < 3; ++axis) {
            double dx = Rc[axis], dy = Rc[3 + axis], dz = Rc[6 + axis];
            double du = (dx - nx * dz) * iz, dv = (dy - ny * dz) * iz;
            double djx = (nx >= -lx && nx <= lx) ? du : 0, djy = (ny >= -ly && ny <= ly) ? dv : 0;
            double dP[6] = {-cam->fx * dz * iz * iz, 0, -cam->fx * (djx - jx * dz * iz) * iz,
                            0, -cam->fy * dz * iz * iz, -cam->fy * (djy - jy * dz * iz) * iz};
            double daa = 0, dab = 0, dcc = 0;
            for (int j = 0; j < 3; ++j) {
                daa += 2 * dP[j] * PV[j];
                dab += dP[j] * PV[3 + j] + dP[3 + j] * PV[j];
                dcc += 2 * dP[3 + j] * PV[3 + j];
            }
            double g = in[0] * cam->fx * du + in[1] * cam->fy * dv + in[2] * daa + in[3] * dab + in[4] * dcc;
            for (int ch = 0; ch < 3; ++ch)
                if (color[ch] >= 0) g += in[6 + ch] * dcol[ch][axis];
            grad58[axis * N + id] = g;
            double a = LP[axis], b = LP[3 + axis];
            grad58[(3 + axis) * N + id] = 2 * s2[axis] * (in[2] * a * a + in[3] * a * b + in[4] * b * b);
            int j = (axis + 1) % 3, k = (axis + 2) % 3;
            right[axis] = (s2[j] - s2[k]) * (2 * in[2] * LP[j] * LP[k] + in[3] * (LP[j] * LP[3 + k] + LP[k] * LP[3 + j]) +
                                             2 * in[4] * LP[3 + j] * LP[3 + k]);
        }
        /* axis-angle: g_omega = J_r(omega)^T g_right, J_r^T = I + a [w]x + b [w]x^2 */
        double th2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
        double ca, cb;
        if (th2 > 1e-4) {
            double th = sqrt(th2);
            ca = (1 - cos(th)) / th2;
            cb = (th - sin(th)) / (th2 * th);
        } else {
            ca = 0.5 - th2 / 24.0;
            cb = 1.0 / 6.0 - th2 / 120.0;
        }
        double cr[3];
        for (int axis = 0; axis < 3; ++axis) {
            int j = (axis + 1) % 3, k = (axis + 2) % 3;
            cr[axis] = w[j] * right[k] - w[k] * right[j];
        }
        for (int axis = 0; axis < 3; ++axis) {
            int j = (axis + 1) % 3, k = (axis + 2) % 3;
            grad58[(6 + axis) * N + id] = right[axis] + ca * cr[axis] + cb * (w[j] * cr[k] - w[k] * cr[j]);
        }
        grad58[9 * N + id] = in[5];
        for (int ch = 0; ch < 3; ++ch)
            for (int k = 0; k < K; ++k)
                grad58[(GSN_SH_INDEX + ch * 16 + k) * N + id] = color[ch] >= 0 ? in[6 + ch] * basis[k] : 0;
    }
}

/* solver.cu:651-689 with the bias corrections of solver.cu:912-914. */
void orc_adam(double* params, double* m, double* v, const double* grad58, int n, const orc_lr* lr, uint64_t step) {
    const int64_t N = n;
    double c1 = 1.0 / (1.0 - pow(0.9, (double)step));
    double c2 = 1.0 / (1.0 - pow(0.999, (double)step));
#pragma omp parallel for schedule(static)
    for (int row = 0; row < 58; ++row) {
        double rate = row < 3 ? lr->position
                              : row < 6 ? lr->scale
                                        : row < 9 ? lr->rotation
                                                  : row < 10 ? lr->opacity
                                                             : ((row - 10) % 16 == 0 ? lr->sh_dc : lr->sh_rest);
        for (int64_t i = 0; i < N; ++i) {
            int64_t k = row * N + i;
            double g = grad58[k];
            m[k] = 0.9 * m[k] + 0.1 * g;
            v[k] = 0.999 * v[k] + 0.001 * g * g;
            params[k] -= rate * (m[k] * c1) / (sqrt(v[k] * c2) + 1e-15);
        }
    }
}

/* ------------------------------------------------------------ density */
/* density_controller.cu:60-116, evaluated in float like the reference so the
 * threshold decisions coincide. */
void orc_density_counts(const float* params, int n, const float* gradient_sums, const float* absolute_sums,
                        const uint32_t* observation_counts, float gradient_threshold, float split_threshold,
                        float min_opacity, float max_world_size, int prune_large,
                        float absolute_gradient_threshold, int* out4) {
    const int64_t N = n;
    for (int id = 0; id < n; ++id) {
        float opacity = 1.0f / (1.0f + expf(-params[9 * N + id]));
        float gradient = observation_counts[id] ? gradient_sums[id] / (float)observation_counts[id] : 0.0f;
        if (isnan(gradient)) gradient = 0.0f;
        float s[3];
        for (int a = 0; a < 3; ++a) s[a] = expf(params[(3 + a) * N + id]);
        float max_scale = fmaxf(s[0], fmaxf(s[1], s[2]));
        if (isnan(s[0]) || isnan(s[1]) || isnan(s[2])) max_scale = NAN;
        int selected = gradient >= gradient_threshold;
        int clone = selected && max_scale <= split_threshold;
        float abs_gradient = observation_counts[id] ? absolute_sums[id] / (float)observation_counts[id] : 0.0f;
        int split_selected = absolute_gradient_threshold > 0.0f ? abs_gradient >= absolute_gradient_threshold : selected;
        int split = split_selected && max_scale > split_threshold;
        float remaining = max_scale;
        if (split && prune_large) {
            float x = expf(logf(s[0] / 1.6f)), y = expf(logf(s[1] / 1.6f)), z = expf(logf(s[2] / 1.6f));
            remaining = fmaxf(x, fmaxf(y, z));
            if (isnan(x) || isnan(y) || isnan(z)) remaining = NAN;
        }
        int remove = opacity < min_opacity || (prune_large && remaining > max_world_size);
        out4[4 * id + 0] = !split && !remove;
        out4[4 * id + 1] = clone && !remove;
        out4[4 * id + 2] = split;
        out4[4 * id + 3] = split && !remove;
    }
}

/* density_controller.cu:118-278: survivors, then clones, then the first split
 * child of every kept split, then the second; split children move by
 * R (n * s) and take log(s / 1.6). */
int orc_density_apply(const float* params, int n, const int* c4, const float* samples, float* out, int* parent_ids,
                      int* history_parent_ids) {
    const int64_t N = n;
    int* off = (int*)malloc(sizeof(int) * 4 * (size_t)(n + 1));
    int run[4] = {0, 0, 0, 0};
    for (int i = 0; i <= n; ++i)
        for (int k = 0; k < 4; ++k) {
            off[4 * i + k] = run[k];
            if (i < n) run[k] += c4[4 * i + k];
        }
    int S = run[0], Cn = run[1], Z = run[2], K = run[3];
    int M = S + Cn + 2 * K;
    for (int id = 0; id < n; ++id) {
        const int* c = c4 + 4 * id;
        const int* o = off + 4 * id;
        int split = c[3] != 0;
        if (!c[0] && !c[1] && !split) continue;
        double s[3] = {0, 0, 0}, R[9];
        if (split) {
            for (int a = 0; a < 3; ++a) s[a] = exp((double)params[(3 + a) * N + id]);
            rotation_matrix(params[6 * N + id], params[7 * N + id], params[8 * N + id], R);
        }
        int children = split ? 2 : c[0] + c[1];
        for (int child = 0; child < children; ++child) {
            int dest = split ? S + Cn + child * K + o[3] : ((child == 0 && c[0]) ? o[0] : S + o[1]);
            for (int p = 0; p < 58; ++p) {
                double value = params[p * N + id];
                if (split && p < 3) {
                    double delta = 0;
                    for (int a = 0; a < 3; ++a) {
                        int64_t sample = ((int64_t)child * Z + o[2]) * 3 + a;
                        delta += R[p * 3 + a] * samples[sample] * s[a];
                    }
                    value += delta;
                } else if (split && p >= 3 && p < 6) {
                    value = log(s[p - 3] / 1.6);
                }
                out[(int64_t)p * M + dest] = (float)value;
            }
            if (parent_ids) parent_ids[dest] = id;
            if (history_parent_ids) history_parent_ids[dest] = (!split && child == 0 && c[0]) ? id : -1;
        }
    }
    free(off);
    return M;
}

/* ------------------------------------------------------------ KNN */
/* Exhaustive FP64 search of knn_test.cu:23-32 (plus the neighbour indices). */
void orc_knn3(const float* pts, int n, double* mean_dist2, int* nb) {
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
        double best[3] = {INFINITY, INFINITY, INFINITY};
        int bi[3] = {-1, -1, -1};
        for (int j = 0; j < n; ++j) {
            if (j == i) continue;
            double dx = (double)pts[3 * i] - pts[3 * j], dy = (double)pts[3 * i + 1] - pts[3 * j + 1],
                   dz = (double)pts[3 * i + 2] - pts[3 * j + 2];
            double d = dx * dx + dy * dy + dz * dz;
            if (d < best[2] || (d == best[2] && j < bi[2])) {
                int k = 2;
                while (k > 0 && (d < best[k - 1] || (d == best[k - 1] && j < bi[k - 1]))) {
                    best[k] = best[k - 1];
                    bi[k] = bi[k - 1];
                    --k;
                }
                best[k] = d;
                bi[k] = j;
            }
        }
        int found = n - 1 < 3 ? n - 1 : 3;
        double s = 0;
        for (int k = 0; k < found; ++k) s += best[k];
        mean_dist2[i] = found > 0 ? s / found : 0.0;
        if (nb)
            for (int k = 0; k < 3; ++k) nb[3 * i + k] = k < found ? bi[k] : -1;
    }
}
