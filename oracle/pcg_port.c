/*
 * pcg_port.c — multi-threaded FP32 CPU port of the hot path (test and CPU
 * reference-timing infrastructure; only the cpu_baseline leg and the
 * reference arm of bench.py time it, and tests check it against the oracle).
 *
 * The arithmetic is the reference's FP32 shader math:
 *   sweeps       shaders/diffusion_2d.metal:28-292 (extended to z, 3-D rule
 *                as in pcg_oracle.h), with the per-line Thomas constants
 *                (c' and 1/denominator, identical for every line of one
 *                substrate and axis) hoisted out of the line loop;
 *   Dirichlet    src/microenvironment.mm:127-152 (six faces in 3-D);
 *   secretion    src/cell_phenotype.cpp:526-564 (FP64 per cell, ascending);
 *   mechanics    shaders/mechanics.metal:41-216, shaders/integrate.metal:31-80.
 * Lines are parallel over OpenMP threads; the y and z sweeps walk a whole
 * slab of columns at once (loop interchange) so the inner loop is
 * contiguous and vectorises.
 */
#include "pcg_oracle.h"

#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { float c, fold; float* cp; float* inv; int n; int dir; float T; } line_rule;

/* Per-line constants in double, stored FP32 (same recurrence as the
 * reference's c_prime/denominator sequence). */
static void build_rule(line_rule* r, int n, double c, double hd, int dir, float T)
{
    r->n = n; r->dir = dir; r->T = T; r->c = (float)c;
    r->fold = dir ? (float)(c * (double)T) : 0.0f;
    r->cp = (float*)calloc((size_t)n + 2, sizeof(float));
    r->inv = (float*)calloc((size_t)n + 2, sizeof(float));
    if (n < 3) return;
    const double b_int = 1.0 + 2.0 * c + hd, b_bnd = 1.0 + c + hd;
    if (n == 3) { r->inv[1] = (float)(1.0 / b_int); r->fold = dir ? (float)(2.0 * c * T) : 0.0f; return; }
    double cp = -c / b_bnd;
    r->cp[1] = (float)cp; r->inv[1] = (float)(1.0 / b_bnd);
    for (int i = 2; i < n - 2; i++) {
        double den = b_int + c * cp;
        cp = -c / den;
        r->cp[i] = (float)cp; r->inv[i] = (float)(1.0 / den);
    }
    r->inv[n - 2] = (float)(1.0 / (b_bnd + c * cp));
}

static void free_rule(line_rule* r) { free(r->cp); free(r->inv); }

static void rule_for(line_rule* r, const or_grid* g, const or_substrate* sp, int axis)
{
    const int d = g->nz > 1 ? 3 : 2;
    const float h = axis == 0 ? g->dx : (axis == 1 ? g->dy : g->dz);
    const int n = axis == 0 ? (int)g->nx : (axis == 1 ? (int)g->ny : (int)g->nz);
    const double c = (double)sp->diffusion_coefficient * (double)g->dt / ((double)h * (double)h);
    const double hd = (double)sp->decay_rate * (double)g->dt / (double)d;
    build_rule(r, n, c, hd, sp->dirichlet_enabled != 0, sp->target_value);
}

/* contiguous line (x sweep) */
static void solve_contig(float* v, const line_rule* r)
{
    const int n = r->n;
    if (r->dir) { v[0] = r->T; v[n - 1] = r->T; }
    if (n <= 2) return;
    if (n == 3) { v[1] = (v[1] + r->fold) * r->inv[1]; return; }
    const float c = r->c;
    float d = (v[1] + r->fold) * r->inv[1];
    v[1] = d;
    for (int i = 2; i < n - 2; i++) { d = (v[i] + c * d) * r->inv[i]; v[i] = d; }
    v[n - 2] = (v[n - 2] + r->fold + c * d) * r->inv[n - 2];
    for (int i = n - 3; i >= 1; i--) v[i] = v[i] - r->cp[i] * v[i + 1];
}

/* W adjacent columns with element stride 'st' (y / z sweeps) */
static void solve_cols(float* base, size_t st, size_t W, const line_rule* r)
{
    const int n = r->n;
    if (r->dir) for (size_t w = 0; w < W; w++) { base[w] = r->T; base[(size_t)(n - 1) * st + w] = r->T; }
    if (n <= 2) return;
    float* row1 = base + st;
    if (n == 3) { for (size_t w = 0; w < W; w++) row1[w] = (row1[w] + r->fold) * r->inv[1]; return; }
    const float c = r->c, f = r->fold;
    for (size_t w = 0; w < W; w++) row1[w] = (row1[w] + f) * r->inv[1];
    for (int i = 2; i < n - 2; i++) {
        float* cur = base + (size_t)i * st; const float* prv = cur - st; const float inv = r->inv[i];
        for (size_t w = 0; w < W; w++) cur[w] = (cur[w] + c * prv[w]) * inv;
    }
    {
        float* cur = base + (size_t)(n - 2) * st; const float* prv = cur - st; const float inv = r->inv[n - 2];
        for (size_t w = 0; w < W; w++) cur[w] = (cur[w] + f + c * prv[w]) * inv;
    }
    for (int i = n - 3; i >= 1; i--) {
        float* cur = base + (size_t)i * st; const float* nxt = cur + st; const float cp = r->cp[i];
        for (size_t w = 0; w < W; w++) cur[w] = cur[w] - cp * nxt[w];
    }
}

void port_diffusion_sweeps(float* density, const or_grid* g, const or_substrate* subs)
{
    const size_t nx = g->nx, ny = g->ny, nz = g->nz, nvox = nx * ny * nz;
    for (uint32_t s = 0; s < g->n_substrates; s++) {
        float* base = density + s * nvox;
        line_rule rx, ry, rz;
        rule_for(&rx, g, &subs[s], 0);
        rule_for(&ry, g, &subs[s], 1);
        long long lines = (long long)(ny * nz);
        #pragma omp parallel for schedule(static)
        for (long long l = 0; l < lines; l++) solve_contig(base + (size_t)l * nx, &rx);
        #pragma omp parallel for schedule(static)
        for (long long k = 0; k < (long long)nz; k++) solve_cols(base + (size_t)k * nx * ny, nx, nx, &ry);
        if (nz > 1) {
            rule_for(&rz, g, &subs[s], 2);
            #pragma omp parallel for schedule(static)
            for (long long j = 0; j < (long long)ny; j++) solve_cols(base + (size_t)j * nx, nx * ny, nx, &rz);
            free_rule(&rz);
        }
        free_rule(&rx); free_rule(&ry);
    }
}

void port_apply_dirichlet(float* density, const or_grid* g, const or_substrate* subs)
{
    or_apply_dirichlet(density, g, subs);
}

void port_secretion(float* density, const or_grid* g, uint32_t n_cells,
                    const uint32_t* voxel, const float* volume,
                    const double* secretion, const double* uptake,
                    const double* saturation, const double* net_export,
                    const uint8_t* active, double dt)
{
    or_secretion(density, g, n_cells, voxel, volume, secretion, uptake, saturation, net_export, active, dt);
}

static int trunc_sat(float q)
{
    if (q != q) return 0;
    if (q >= 2147483648.0f) return INT_MAX;
    if (q <= -2147483648.0f) return INT_MIN;
    return (int)q;
}
static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* One mechanics step: bin, counting sort, forces, AB2 integrate. */
void port_mech_step(float* soa, uint32_t max_cells, uint32_t n_cells, const or_mech* m,
                    float x_min, float y_min, float z_min, float dt,
                    uint32_t* key, uint32_t* order, uint32_t* start)
{
    float* px = soa + (size_t)OR_F_POS_X * max_cells;
    float* py = soa + (size_t)OR_F_POS_Y * max_cells;
    float* pz = soa + (size_t)OR_F_POS_Z * max_cells;
    float* vx = soa + (size_t)OR_F_VEL_X * max_cells;
    float* vy = soa + (size_t)OR_F_VEL_Y * max_cells;
    float* vz = soa + (size_t)OR_F_VEL_Z * max_cells;
    float* pvx = soa + (size_t)OR_F_PREV_VX * max_cells;
    float* pvy = soa + (size_t)OR_F_PREV_VY * max_cells;
    float* pvz = soa + (size_t)OR_F_PREV_VZ * max_cells;
    const float* rad = soa + (size_t)OR_F_RADIUS * max_cells;
    const float* rep = soa + (size_t)OR_F_REPULSION * max_cells;
    const float* adh = soa + (size_t)OR_F_ADHESION * max_cells;
    const float* rel = soa + (size_t)OR_F_REL_MAX_ADH * max_cells;
    float* pr = soa + (size_t)OR_F_PRESSURE * max_cells;
    uint32_t* mv = (uint32_t*)(soa + (size_t)OR_F_MECH_VOXEL * max_cells);
    const uint32_t mnx = m->mech_grid_nx, mny = m->mech_grid_ny, mnz = m->mech_grid_nz;
    const uint32_t V = mnx * mny * mnz;
    const float vs = m->mechanics_voxel_size;
    #pragma omp parallel for schedule(static)
    for (long long t = 0; t < (long long)n_cells; t++) {
        int vi = clampi(trunc_sat((px[t] - x_min) / vs), 0, (int)mnx - 1);
        int vj = clampi(trunc_sat((py[t] - y_min) / vs), 0, (int)mny - 1);
        int vk = clampi(trunc_sat((pz[t] - z_min) / vs), 0, (int)mnz - 1);
        uint32_t v = (uint32_t)vk * mny * mnx + (uint32_t)vj * mnx + (uint32_t)vi;
        key[t] = v; mv[t] = v;
    }
    memset(start, 0, sizeof(uint32_t) * ((size_t)V + 1));
    for (uint32_t i = 0; i < n_cells; i++) start[key[i] + 1]++;
    for (uint32_t v = 0; v < V; v++) start[v + 1] += start[v];
    {
        uint32_t* fill = (uint32_t*)malloc(sizeof(uint32_t) * ((size_t)V + 1));
        memcpy(fill, start, sizeof(uint32_t) * ((size_t)V + 1));
        for (uint32_t i = 0; i < n_cells; i++) order[fill[key[i]]++] = i;
        free(fill);
    }
    const float maxd = m->max_interaction_distance;
    float* out = (float*)malloc(sizeof(float) * 4 * (n_cells ? n_cells : 1));
    #pragma omp parallel for schedule(dynamic, 256)
    for (long long ii = 0; ii < (long long)n_cells; ii++) {
        uint32_t i = (uint32_t)ii;
        float xi = px[i], yi = py[i], zi = pz[i], Ri = rad[i], rpi = rep[i], adi = adh[i], rmi = rel[i];
        uint32_t my = key[i];
        uint32_t ci = my % mnx, cj = (my / mnx) % mny, ck = my / (mnx * mny);
        int dkmin = mnz > 1 ? -1 : 0, dkmax = mnz > 1 ? 1 : 0;
        float fx = 0, fy = 0, fz = 0, P = 0;
        for (int dk = dkmin; dk <= dkmax; dk++) {
            int nk = (int)ck + dk;
            if (nk < 0 || nk >= (int)mnz) continue;
            for (int dj = -1; dj <= 1; dj++) {
                int nj = (int)cj + dj;
                if (nj < 0 || nj >= (int)mny) continue;
                int ilo = (int)ci > 0 ? (int)ci - 1 : 0, ihi = (int)ci + 1 < (int)mnx ? (int)ci + 1 : (int)mnx - 1;
                uint32_t row = (uint32_t)nk * mny * mnx + (uint32_t)nj * mnx;
                for (uint32_t q = start[row + ilo]; q < start[row + ihi + 1]; q++) {
                    uint32_t j = order[q];
                    if (j == i) continue;
                    float ddx = xi - px[j], ddy = yi - py[j], ddz = zi - pz[j];
                    float dsq = ddx * ddx + ddy * ddy + ddz * ddz;
                    if (dsq >= maxd * maxd || dsq < 1e-12f) continue;
                    float dist = sqrtf(dsq), inv = 1.0f / dist;
                    float R = Ri + rad[j], F = 0.0f;
                    if (dist < R) {
                        float ov = 1.0f - dist / R;
                        F += ov * ov * sqrtf(rpi * rep[j]);
                        P += ov * ov / 0.027288820670331f;
                    }
                    float A = rmi * R;
                    if (dist < A) { float t = 1.0f - dist / A; F -= t * t * sqrtf(adi * adh[j]); }
                    fx += F * ddx * inv; fy += F * ddy * inv; fz += F * ddz * inv;
                }
            }
        }
        out[4 * i] = fx; out[4 * i + 1] = fy; out[4 * i + 2] = fz; out[4 * i + 3] = P;
    }
    const float xmax = x_min + (float)mnx * vs, ymax = y_min + (float)mny * vs, zmax = z_min + (float)mnz * vs;
    #pragma omp parallel for schedule(static)
    for (long long t = 0; t < (long long)n_cells; t++) {
        float fx = out[4 * t], fy = out[4 * t + 1], fz = out[4 * t + 2];
        vx[t] = fx; vy[t] = fy; vz[t] = fz; pr[t] = out[4 * t + 3];
        float x = px[t] + dt * (1.5f * fx - 0.5f * pvx[t]);
        float y = py[t] + dt * (1.5f * fy - 0.5f * pvy[t]);
        float z = pz[t] + dt * (1.5f * fz - 0.5f * pvz[t]);
        px[t] = fminf(fmaxf(x, x_min), xmax);
        py[t] = fminf(fmaxf(y, y_min), ymax);
        pz[t] = fminf(fmaxf(z, z_min), zmax);
        pvx[t] = fx; pvy[t] = fy; pvz[t] = fz;
    }
    free(out);
}

int port_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void port_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
