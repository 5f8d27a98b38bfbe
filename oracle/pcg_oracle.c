/*
 * pcg_oracle.c — CPU oracle for the per-step hot path (TEST INFRASTRUCTURE).
 * See pcg_oracle.h for scope, precision modes and the determinism rules.
 * Build with -ffp-contract=off: the FP32 paths must be the plain IEEE
 * operation sequence of the reference source.
 */
#include "pcg_oracle.h"

#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* Diffusion                                                           */
/* ------------------------------------------------------------------ */

/* Line solve in double, following diffusion_2d.metal:55-155 (x sweep; the y
 * sweep :196-290 is the same rule along another axis).  v holds the n values
 * of the line; cp is scratch of n doubles. */
static void solve_line_f64(double* v, double* cp, int n, double c, double hd, int dir, double T, int consistent)
{
    const double b_int = 1.0 + 2.0 * c + hd;   /* :47 */
    /* :48; the consistent Dirichlet option gives the end interior nodes of a
     * Dirichlet line the interior diagonal */
    const double b_bnd = (dir && consistent) ? b_int : 1.0 + c + hd;
    if (dir) { v[0] = T; v[n - 1] = T; }       /* :55-58 */
    if (n <= 2) return;                        /* :60-63 */
    if (n == 3) {                              /* :66-84: b_int, both folds */
        double d = v[1];
        if (dir) { d += c * T; d += c * T; }
        v[1] = d / b_int;
    } else {
        /* first interior node, boundary diagonal, fold c*T (:90-108) */
        double d = v[1];
        if (dir) d += c * T;
        double cprev = -c / b_bnd;
        double dprev = d / b_bnd;
        cp[1] = cprev;
        v[1] = dprev;
        /* inner nodes (:111-124): a = c_i = -c, b = b_int */
        for (int i = 2; i < n - 2; i++) {
            double den = b_int + c * cprev;
            cprev = -c / den;
            dprev = (v[i] + c * dprev) / den;
            cp[i] = cprev;
            v[i] = dprev;
        }
        /* last interior node, boundary diagonal, fold c*T (:127-142) */
        {
            double dl = v[n - 2];
            if (dir) dl += c * T;
            double den = b_bnd + c * cprev;
            v[n - 2] = (dl + c * dprev) / den;
        }
        /* back substitution (:145-148) */
        for (int i = n - 3; i >= 1; i--) v[i] = v[i] - cp[i] * v[i + 1];
    }
    if (dir) { v[0] = T; v[n - 1] = T; }       /* :152-155 */
}

/* The same rule as the reference writes it in FP32 (every operation rounded
 * to float, in the source's order, in-place d' storage). */
static void solve_line_f32(float* v, float* cp, int n, float coeff, float half_decay, int dir, float target)
{
    const float diag_interior = 1.0f + 2.0f * coeff + half_decay;
    const float diag_boundary = 1.0f + coeff + half_decay;
    if (dir) { v[0] = target; v[n - 1] = target; }
    if (n <= 2) return;
    if (n == 3) {
        float d_i = v[1];
        float b = diag_interior;
        if (dir) { d_i += coeff * target; d_i += coeff * target; }
        v[1] = d_i / b;
        if (dir) { v[0] = target; v[n - 1] = target; }
        return;
    }
    {
        float d_i = v[1];
        float b_1 = diag_boundary;
        float c_1 = -coeff;
        if (dir) d_i += coeff * target;
        float c_p = c_1 / b_1;
        float d_p = d_i / b_1;
        cp[1] = c_p;
        v[1] = d_p;
        float c_prev = c_p, d_prev = d_p;
        for (int i = 2; i < n - 2; i++) {
            float a_i = -coeff, b_i = diag_interior, c_i = -coeff;
            d_i = v[i];
            float denom = b_i - a_i * c_prev;
            c_prev = c_i / denom;
            d_prev = (d_i - a_i * d_prev) / denom;
            cp[i] = c_prev;
            v[i] = d_prev;
        }
        {
            float a_last = -coeff, b_last = diag_boundary;
            d_i = v[n - 2];
            if (dir) d_i += coeff * target;
            float denom = b_last - a_last * c_prev;
            d_prev = (d_i - a_last * d_prev) / denom;
            v[n - 2] = d_prev;
        }
        for (int i = n - 3; i >= 1; i--) v[i] = v[i] - cp[i] * v[i + 1];
    }
    if (dir) { v[0] = target; v[n - 1] = target; }
}

static int n_sweeps(const or_grid* g) { return g->nz > 1 ? 3 : 2; }

void or_sweep_axis(float* density, const or_grid* g, const or_substrate* subs, int axis, int mode)
{
    const size_t nx = g->nx, ny = g->ny, nz = g->nz;
    const size_t nvox = nx * ny * nz;
    size_t n, stride, lines_a, lines_b, stride_a, stride_b;
    float h;
    if (axis == 0) {        /* lines along i; families over (j, k) */
        n = nx; stride = 1; lines_a = ny; stride_a = nx; lines_b = nz; stride_b = nx * ny; h = g->dx;
    } else if (axis == 1) { /* lines along j; families over (i, k) */
        n = ny; stride = nx; lines_a = nx; stride_a = 1; lines_b = nz; stride_b = nx * ny; h = g->dy;
    } else {                /* lines along k; families over (i, j) */
        n = nz; stride = nx * ny; lines_a = nx; stride_a = 1; lines_b = ny; stride_b = nx; h = g->dz;
    }
    if (n == 0) return;
    const int d = n_sweeps(g);
    double* vd = (double*)malloc(sizeof(double) * (n + 2));
    double* cd = (double*)malloc(sizeof(double) * (n + 2));
    float* vf = (float*)malloc(sizeof(float) * (n + 2));
    float* cf = (float*)malloc(sizeof(float) * (n + 2));
    for (uint32_t s = 0; s < g->n_substrates; s++) {
        const or_substrate* sp = &subs[s];
        const int dir = sp->dirichlet_enabled != 0;
        /* coefficient D*dt/h^2 (microenvironment.mm:90, diffusion_2d.metal:181-184) */
        const double c64 = (double)sp->diffusion_coefficient * (double)g->dt / ((double)h * (double)h);
        const double hd64 = (double)sp->decay_rate * (double)g->dt / (double)d;
        const float D = sp->diffusion_coefficient, dt = g->dt;
        const float c32 = D * dt / (h * h);
        const float hd32 = (d == 2) ? 0.5f * sp->decay_rate * dt : sp->decay_rate * dt / 3.0f;
        float* base = density + s * nvox;
        for (size_t b = 0; b < lines_b; b++) {
            for (size_t a = 0; a < lines_a; a++) {
                float* line = base + a * stride_a + b * stride_b;
                if (mode == OR_FP32_REF) {
                    for (size_t m = 0; m < n; m++) vf[m] = line[m * stride];
                    solve_line_f32(vf, cf, (int)n, c32, hd32, dir, sp->target_value);
                    for (size_t m = 0; m < n; m++) line[m * stride] = vf[m];
                } else {
                    for (size_t m = 0; m < n; m++) vd[m] = (double)line[m * stride];
                    solve_line_f64(vd, cd, (int)n, c64, hd64, dir, (double)sp->target_value,
                                   sp->dirichlet_consistent != 0);
                    for (size_t m = 0; m < n; m++) line[m * stride] = (float)vd[m];
                }
            }
        }
    }
    free(vd); free(cd); free(vf); free(cf);
}

void or_diffusion_sweeps(float* density, const or_grid* g, const or_substrate* subs, int mode)
{
    or_sweep_axis(density, g, subs, 0, mode);
    or_sweep_axis(density, g, subs, 1, mode);
    if (g->nz > 1) or_sweep_axis(density, g, subs, 2, mode);
}

void or_apply_dirichlet(float* density, const or_grid* g, const or_substrate* subs)
{
    const size_t nx = g->nx, ny = g->ny, nz = g->nz, nvox = nx * ny * nz;
    if (nx == 0 || ny == 0 || nz == 0) return;
    for (uint32_t s = 0; s < g->n_substrates; s++) {
        if (!subs[s].dirichlet_enabled) continue;
        const float T = subs[s].target_value;
        float* base = density + s * nvox;
        for (size_t k = 0; k < nz; k++) {
            float* slab = base + k * nx * ny;
            if (nz > 1 && (k == 0 || k == nz - 1)) {  /* z faces (3-D rule) */
                for (size_t v = 0; v < nx * ny; v++) slab[v] = T;
                continue;
            }
            /* microenvironment.mm:140-150 */
            for (size_t i = 0; i < nx; i++) { slab[i] = T; slab[(ny - 1) * nx + i] = T; }
            for (size_t j = 0; j < ny; j++) { slab[j * nx] = T; slab[j * nx + nx - 1] = T; }
        }
    }
}

void or_gradients(const float* density, const or_grid* g, float* gx, float* gy, float* gz)
{
    const size_t nx = g->nx, ny = g->ny, nz = g->nz, nvox = nx * ny * nz;
    const double idx = 1.0 / g->dx, idy = 1.0 / g->dy, idz = 1.0 / g->dz;
    for (uint32_t s = 0; s < g->n_substrates; s++) {
        const float* D = density + s * nvox;
        for (size_t k = 0; k < nz; k++)
            for (size_t j = 0; j < ny; j++)
                for (size_t i = 0; i < nx; i++) {
                    size_t n = k * nx * ny + j * nx + i, o = s * nvox + n;
                    double v;
                    if (nx == 1) v = 0.0;
                    else if (i == 0) v = ((double)D[n + 1] - D[n]) * idx;
                    else if (i == nx - 1) v = ((double)D[n] - D[n - 1]) * idx;
                    else v = ((double)D[n + 1] - D[n - 1]) * 0.5 * idx;
                    gx[o] = (float)v;
                    if (ny == 1) v = 0.0;
                    else if (j == 0) v = ((double)D[n + nx] - D[n]) * idy;
                    else if (j == ny - 1) v = ((double)D[n] - D[n - nx]) * idy;
                    else v = ((double)D[n + nx] - D[n - nx]) * 0.5 * idy;
                    gy[o] = (float)v;
                    if (nz > 1) {
                        size_t sz = nx * ny;
                        if (k == 0) v = ((double)D[n + sz] - D[n]) * idz;
                        else if (k == nz - 1) v = ((double)D[n] - D[n - sz]) * idz;
                        else v = ((double)D[n + sz] - D[n - sz]) * 0.5 * idz;
                    } else v = 0.0;
                    gz[o] = (float)v;
                }
    }
}

/* ------------------------------------------------------------------ */
/* Secretion (cell_phenotype.cpp:526-564)                              */
/* ------------------------------------------------------------------ */

void or_secretion(float* density, const or_grid* g, uint32_t n_cells,
                  const uint32_t* voxel, const float* volume,
                  const double* secretion, const double* uptake,
                  const double* saturation, const double* net_export,
                  const uint8_t* active, double dt)
{
    const uint32_t S = g->n_substrates;
    if (!density || S == 0) return;
    const uint32_t total = g->nx * g->ny * g->nz;
    const double V_voxel = (double)g->dx * (double)g->dy * (double)g->dz;
    for (uint32_t i = 0; i < n_cells; i++) {
        if (active && !active[i]) continue;
        uint32_t vi = voxel[i];
        if (vi >= total) continue;
        double V_cell = (double)volume[i];
        double ic = dt * V_cell / V_voxel;
        for (uint32_t s = 0; s < S; s++) {
            size_t off = (size_t)i * S + s;
            double sec = secretion[off], upt = uptake[off], sat = saturation[off], ne = net_export[off];
            size_t vo = (size_t)s * total + vi;
            double rho = (double)density[vo];
            rho += dt * ne / V_voxel;
            double t1 = ic * sec * sat;
            double t2 = 1.0 + ic * (sec + upt);
            rho = (rho + t1) / t2;
            if (rho < 0.0) rho = 0.0;
            density[vo] = (float)rho;
        }
    }
}

/* ------------------------------------------------------------------ */
/* Mechanics                                                           */
/* ------------------------------------------------------------------ */

void or_mech_params(float x_min, float x_max, float y_min, float y_max,
                    float z_min, float z_max, int use_2d, float dt_mech, or_mech* m)
{
    /* cell_mechanics.mm:26-41 */
    const float vs = 30.0f;
    float Lx = x_max - x_min, Ly = y_max - y_min, Lz = z_max - z_min;
    uint32_t nx = (uint32_t)(Lx / vs), ny = (uint32_t)(Ly / vs), nz = (uint32_t)(Lz / vs);
    m->dt = dt_mech;
    m->cell_cell_repulsion = 10.0f;
    m->cell_cell_adhesion = 0.4f;
    m->max_interaction_distance = vs;
    m->mechanics_voxel_size = vs;
    m->mech_grid_nx = nx < 1 ? 1 : nx;
    m->mech_grid_ny = ny < 1 ? 1 : ny;
    m->mech_grid_nz = use_2d ? 1 : (nz < 1 ? 1 : nz);
}

/* float -> int truncation with saturation and NaN -> 0 (the behaviour of
 * the GPU's cvt.rzi.s32.f32); the reference relies on in-range values. */
static int trunc_sat(float q)
{
    if (q != q) return 0;
    if (q >= 2147483648.0f) return INT_MAX;
    if (q <= -2147483648.0f) return INT_MIN;
    return (int)q;
}

static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

void or_mech_bin(float* soa, uint32_t max_cells, uint32_t n_cells, const or_mech* m,
                 float x_min, float y_min, float z_min, uint32_t* key)
{
    const float* px = soa + (size_t)OR_F_POS_X * max_cells;
    const float* py = soa + (size_t)OR_F_POS_Y * max_cells;
    const float* pz = soa + (size_t)OR_F_POS_Z * max_cells;
    uint32_t* mv = (uint32_t*)(soa + (size_t)OR_F_MECH_VOXEL * max_cells);
    const float vs = m->mechanics_voxel_size;
    for (uint32_t t = 0; t < n_cells; t++) {
        int vi = trunc_sat((px[t] - x_min) / vs);
        int vj = trunc_sat((py[t] - y_min) / vs);
        int vk = trunc_sat((pz[t] - z_min) / vs);
        vi = clampi(vi, 0, (int)m->mech_grid_nx - 1);
        vj = clampi(vj, 0, (int)m->mech_grid_ny - 1);
        vk = clampi(vk, 0, (int)m->mech_grid_nz - 1);
        uint32_t v = (uint32_t)vk * m->mech_grid_ny * m->mech_grid_nx + (uint32_t)vj * m->mech_grid_nx + (uint32_t)vi;
        key[t] = v;
        mv[t] = v;
    }
}

void or_mech_sort(const uint32_t* key, uint32_t n_cells, uint32_t n_voxels,
                  uint32_t* order, uint32_t* start)
{
    memset(start, 0, sizeof(uint32_t) * ((size_t)n_voxels + 1));
    for (uint32_t i = 0; i < n_cells; i++) start[key[i] + 1]++;
    for (uint32_t v = 0; v < n_voxels; v++) start[v + 1] += start[v];
    uint32_t* fill = (uint32_t*)malloc(sizeof(uint32_t) * ((size_t)n_voxels + 1));
    memcpy(fill, start, sizeof(uint32_t) * ((size_t)n_voxels + 1));
    for (uint32_t i = 0; i < n_cells; i++) order[fill[key[i]]++] = i;  /* ascending i: stable */
    free(fill);
}

uint32_t or_nbr_hash(uint32_t j)
{
    uint32_t x = j + 0x9E3779B9u;
    x ^= x >> 16; x *= 0x85EBCA6Bu;
    x ^= x >> 13; x *= 0xC2B2AE35u;
    x ^= x >> 16;
    return x;
}

void or_mech_forces(float* soa, uint32_t max_cells, uint32_t n_cells, const or_mech* m,
                    const uint32_t* key, const uint32_t* order, const uint32_t* start,
                    uint32_t* nbr_count, uint32_t* nbr_hash, double* force_scale)
{
    const float* px = soa + (size_t)OR_F_POS_X * max_cells;
    const float* py = soa + (size_t)OR_F_POS_Y * max_cells;
    const float* pz = soa + (size_t)OR_F_POS_Z * max_cells;
    const float* rad = soa + (size_t)OR_F_RADIUS * max_cells;
    const float* rep = soa + (size_t)OR_F_REPULSION * max_cells;
    const float* adh = soa + (size_t)OR_F_ADHESION * max_cells;
    const float* rel = soa + (size_t)OR_F_REL_MAX_ADH * max_cells;
    float* vx = soa + (size_t)OR_F_VEL_X * max_cells;
    float* vy = soa + (size_t)OR_F_VEL_Y * max_cells;
    float* vz = soa + (size_t)OR_F_VEL_Z * max_cells;
    float* pr = soa + (size_t)OR_F_PRESSURE * max_cells;
    const uint32_t mnx = m->mech_grid_nx, mny = m->mech_grid_ny, mnz = m->mech_grid_nz;
    const float maxd = m->max_interaction_distance;
    const float maxd2 = maxd * maxd;
    const double pscale = (double)0.027288820670331f;   /* mechanics.metal:188 */
    /* outputs are written after all inputs are read (forces read positions only) */
    float* ox = (float*)malloc(sizeof(float) * (n_cells ? n_cells : 1) * 4);
    for (uint32_t i = 0; i < n_cells; i++) {
        const float xi = px[i], yi = py[i], zi = pz[i];
        const double Ri = rad[i], rpi = rep[i], adi = adh[i], rmi = rel[i];
        uint32_t my = key[i];
        uint32_t ci = my % mnx, cj = (my / mnx) % mny, ck = my / (mnx * mny);
        int dkmin = mnz > 1 ? -1 : 0, dkmax = mnz > 1 ? 1 : 0;
        double fx = 0, fy = 0, fz = 0, P = 0, scale = 0;
        uint32_t cnt = 0, h = 0;
        for (int dk = dkmin; dk <= dkmax; dk++) {
            int nk = (int)ck + dk;
            if (nk < 0 || nk >= (int)mnz) continue;
            for (int dj = -1; dj <= 1; dj++) {
                int nj = (int)cj + dj;
                if (nj < 0 || nj >= (int)mny) continue;
                for (int di = -1; di <= 1; di++) {
                    int ni = (int)ci + di;
                    if (ni < 0 || ni >= (int)mnx) continue;
                    uint32_t nv = (uint32_t)nk * mny * mnx + (uint32_t)nj * mnx + (uint32_t)ni;
                    for (uint32_t q = start[nv]; q < start[nv + 1]; q++) {
                        uint32_t j = order[q];
                        if (j == i) continue;
                        /* FP32 neighbour test exactly as mechanics.metal:159-165 */
                        float ddx = xi - px[j], ddy = yi - py[j], ddz = zi - pz[j];
                        float dsq = ddx * ddx + ddy * ddy + ddz * ddz;
                        if (dsq >= maxd2) continue;
                        if (dsq < 1e-12f) continue;
                        cnt++;
                        h += or_nbr_hash(j);
                        double ex = (double)xi - (double)px[j];
                        double ey = (double)yi - (double)py[j];
                        double ez = (double)zi - (double)pz[j];
                        double dist = sqrt(ex * ex + ey * ey + ez * ez);
                        double R = Ri + (double)rad[j];
                        double F = 0.0;
                        if (dist < R) {
                            double ov = 1.0 - dist / R;
                            double fr = ov * ov * sqrt(rpi * (double)rep[j]);
                            F += fr;
                            scale += fr;
                            P += ov * ov / pscale;
                        }
                        double A = rmi * R;
                        if (dist < A) {
                            double t = 1.0 - dist / A;
                            double fa = t * t * sqrt(adi * (double)adh[j]);
                            F -= fa;
                            scale += fa;
                        }
                        fx += F * (ex / dist);
                        fy += F * (ey / dist);
                        fz += F * (ez / dist);
                    }
                }
            }
        }
        ox[4 * i + 0] = (float)fx; ox[4 * i + 1] = (float)fy;
        ox[4 * i + 2] = (float)fz; ox[4 * i + 3] = (float)P;
        if (nbr_count) nbr_count[i] = cnt;
        if (nbr_hash) nbr_hash[i] = h;
        if (force_scale) force_scale[i] = scale;
    }
    for (uint32_t i = 0; i < n_cells; i++) {
        vx[i] = ox[4 * i]; vy[i] = ox[4 * i + 1]; vz[i] = ox[4 * i + 2]; pr[i] = ox[4 * i + 3];
    }
    free(ox);
}

void or_mech_integrate(float* soa, uint32_t max_cells, uint32_t n_cells, const or_mech* m,
                       float x_min, float y_min, float z_min, float dt)
{
    or_mech_integrate_master(soa, max_cells, n_cells, m, x_min, y_min, z_min, dt, NULL);
}

void or_mech_integrate_master(float* soa, uint32_t max_cells, uint32_t n_cells, const or_mech* m,
                              float x_min, float y_min, float z_min, float dt, double* pos64)
{
    float* p[3] = { soa + (size_t)OR_F_POS_X * max_cells, soa + (size_t)OR_F_POS_Y * max_cells,
                    soa + (size_t)OR_F_POS_Z * max_cells };
    float* v[3] = { soa + (size_t)OR_F_VEL_X * max_cells, soa + (size_t)OR_F_VEL_Y * max_cells,
                    soa + (size_t)OR_F_VEL_Z * max_cells };
    float* pv[3] = { soa + (size_t)OR_F_PREV_VX * max_cells, soa + (size_t)OR_F_PREV_VY * max_cells,
                     soa + (size_t)OR_F_PREV_VZ * max_cells };
    /* clamp box: the mechanics grid's GridParams (cell_mechanics.mm:57-70)
     * as integrate.metal:58-69 clamps to it */
    const float lo[3] = { x_min, y_min, z_min };
    const uint32_t nn[3] = { m->mech_grid_nx, m->mech_grid_ny, m->mech_grid_nz };
    float hi[3];
    for (int a = 0; a < 3; a++) hi[a] = lo[a] + (float)nn[a] * m->mechanics_voxel_size;
    const double ddt = (double)dt;
    for (uint32_t t = 0; t < n_cells; t++) {
        for (int a = 0; a < 3; a++) {
            double vv = (double)v[a][t], pp = (double)pv[a][t];
            double inc = 1.5 * vv - 0.5 * pp;
            double x0 = (double)p[a][t];
            if (pos64) {
                const double mst = pos64[(size_t)a * max_cells + t];
                if ((float)mst == p[a][t]) x0 = mst;
            }
            double x = x0 + ddt * inc;
            if (x < (double)lo[a]) x = lo[a];
            if (x > (double)hi[a]) x = hi[a];
            if (pos64) pos64[(size_t)a * max_cells + t] = x;
            p[a][t] = (float)x;
            pv[a][t] = v[a][t];
        }
    }
}

void or_voxel_refresh(float* soa, uint32_t max_cells, uint32_t n_cells, const or_grid* g)
{
    const float* px = soa + (size_t)OR_F_POS_X * max_cells;
    const float* py = soa + (size_t)OR_F_POS_Y * max_cells;
    const float* pz = soa + (size_t)OR_F_POS_Z * max_cells;
    uint32_t* vox = (uint32_t*)(soa + (size_t)OR_F_VOXEL_IDX * max_cells);
    for (uint32_t t = 0; t < n_cells; t++) {
        int i = clampi(trunc_sat((px[t] - g->x_min) / g->dx), 0, (int)g->nx - 1);
        int j = clampi(trunc_sat((py[t] - g->y_min) / g->dy), 0, (int)g->ny - 1);
        int k = clampi(trunc_sat((pz[t] - g->z_min) / g->dz), 0, (int)g->nz - 1);
        vox[t] = (uint32_t)k * g->nx * g->ny + (uint32_t)j * g->nx + (uint32_t)i;
    }
}

/* ------------------------------------------------------------------ */
/* Dead-cell compaction (cell_phenotype.cpp:838-844, cell_data.cpp:408-498) */
/* ------------------------------------------------------------------ */

static int cmp_desc_u32(const void* a, const void* b)
{
    const uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
    return x < y ? 1 : (x > y ? -1 : 0);
}

uint32_t or_cells_remove(float* soa, uint32_t max_cells, uint32_t n_cells, uint32_t S, double* sec, double* upt,
                         double* sat, double* ne, uint8_t* active, const uint32_t* indices, uint32_t count)
{
    uint32_t* r = (uint32_t*)malloc((count ? count : 1) * sizeof(uint32_t));
    if (!r) return n_cells;
    if (count) memcpy(r, indices, count * sizeof(uint32_t));
    qsort(r, count, sizeof(uint32_t), cmp_desc_u32);
    uint32_t* u = (uint32_t*)soa;
    double* rates[4] = {sec, upt, sat, ne};
    uint32_t num = n_cells;
    for (uint32_t q = 0; q < count; q++) {
        const uint32_t idx = r[q];
        if (idx >= num) continue;
        const uint32_t last = num - 1;
        if (idx != last) {
            for (int f = 0; f < OR_NUM_FIELDS; f++) u[(size_t)f * max_cells + idx] = u[(size_t)f * max_cells + last];
            for (int a = 0; a < 4; a++)
                if (rates[a])
                    for (uint32_t s = 0; s < S; s++) rates[a][(size_t)idx * S + s] = rates[a][(size_t)last * S + s];
            if (active) active[idx] = active[last];
        }
        num--;
    }
    free(r);
    return num;
}

/* ------------------------------------------------------------------ */
/* Whole step (main.mm:341-391)                                         */
/* ------------------------------------------------------------------ */

/* ------------------------------------------------------------------ motility */

#define OR_PI 3.14159265358979323846

static uint64_t or_mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

double or_uniform(uint64_t seed, uint64_t cell, uint64_t step, uint32_t k)
{
    uint64_t h = or_mix64(seed ^ 0x9e3779b97f4a7c15ULL);
    h = or_mix64(h ^ cell);
    h = or_mix64(h ^ step);
    h = or_mix64(h ^ (uint64_t)k);
    return (double)(h >> 11) * 0x1.0p-53;
}

/* The density value at the clamped voxel (i, j, k) for substrate s, read as
 * the reference reads it (layout OR_MOT_REF) or substrate-major. */
static double or_mot_density(const float* density, const or_grid* g, int i, int j, int k, int s, int layout)
{
    const int nx = (int)g->nx, ny = (int)g->ny, nz = (int)g->nz;
    i = i < 0 ? 0 : (i > nx - 1 ? nx - 1 : i);
    j = j < 0 ? 0 : (j > ny - 1 ? ny - 1 : j);
    k = k < 0 ? 0 : (k > nz - 1 ? nz - 1 : k);
    const size_t v = ((size_t)k * ny + j) * nx + i;
    const size_t nvox = (size_t)g->nx * g->ny * g->nz;
    return (double)density[layout == OR_MOT_REF ? v * g->n_substrates + (size_t)s : (size_t)s * nvox + v];
}

/* computeGradient (motility.cpp:46-87): voxel by FP32 subtract and divide,
 * truncation, clamp; central differences with clamped neighbours. */
static void or_mot_gradient(const float* density, const or_grid* g, float px, float py, float pz, int s,
                            int layout, double* gx, double* gy, double* gz)
{
    if (s < 0 || s >= (int)g->n_substrates) {   /* undefined in the reference: no gradient */
        *gx = *gy = *gz = 0.0;
        return;
    }
    const int nx = (int)g->nx, ny = (int)g->ny, nz = (int)g->nz;
    int ix = (int)((px - g->x_min) / g->dx);
    int iy = (int)((py - g->y_min) / g->dy);
    int iz = (int)((pz - g->z_min) / g->dz);
    ix = ix < 0 ? 0 : (ix > nx - 1 ? nx - 1 : ix);
    iy = iy < 0 ? 0 : (iy > ny - 1 ? ny - 1 : iy);
    iz = iz < 0 ? 0 : (iz > nz - 1 ? nz - 1 : iz);
    *gx = (or_mot_density(density, g, ix + 1, iy, iz, s, layout) - or_mot_density(density, g, ix - 1, iy, iz, s, layout)) /
          (2.0 * g->dx);
    *gy = (or_mot_density(density, g, ix, iy + 1, iz, s, layout) - or_mot_density(density, g, ix, iy - 1, iz, s, layout)) /
          (2.0 * g->dy);
    *gz = 0.0;
    if (nz > 1)
        *gz = (or_mot_density(density, g, ix, iy, iz + 1, s, layout) -
               or_mot_density(density, g, ix, iy, iz - 1, s, layout)) /
              (2.0 * g->dz);
}

void or_motility_update(float* soa, uint32_t max_cells, uint32_t n_cells, const float* density,
                        const or_grid* g, or_motility* m, double dt, uint64_t seed, uint64_t step, int layout)
{
    float* px = soa + (size_t)0 * max_cells;
    float* py = soa + (size_t)1 * max_cells;
    float* pz = soa + (size_t)2 * max_cells;
    float* vx = soa + (size_t)3 * max_cells;
    float* vy = soa + (size_t)4 * max_cells;
    float* vz = soa + (size_t)5 * max_cells;
    const float* speed = soa + (size_t)16 * max_cells;
    const float* alive = soa + (size_t)25 * max_cells;
    double* mvx = m->vec;
    double* mvy = m->vec + n_cells;
    double* mvz = m->vec + 2 * (size_t)n_cells;
    for (uint32_t i = 0; i < n_cells; i++) {
        uint32_t is_alive;
        memcpy(&is_alive, &alive[i], sizeof is_alive);
        if (is_alive == 0) continue;
        if (m->is_motile[i] == 0) {
            mvx[i] = mvy[i] = mvz[i] = 0.0;
            continue;
        }
        m->elapsed[i] += dt;
        const double pt = m->persistence_time[i];
        const int resample = (pt < dt) || (or_uniform(seed, i, step, 0) < dt / pt);
        if (resample) {
            m->elapsed[i] = 0.0;
            double rx, ry, rz;
            if (m->restrict_2d[i]) {
                const double theta = 2.0 * OR_PI * or_uniform(seed, i, step, 1);
                rx = cos(theta);
                ry = sin(theta);
                rz = 0.0;
            } else {
                const double theta = 2.0 * OR_PI * or_uniform(seed, i, step, 1);
                const double phi = OR_PI * or_uniform(seed, i, step, 2);
                const double sin_phi = sin(phi);
                rx = sin_phi * cos(theta);
                ry = sin_phi * sin(theta);
                rz = cos(phi);
            }
            double bx = 0.0, by = 0.0, bz = 0.0;
            const double bias = m->bias[i];
            if (bias > 0.0 && density != NULL) {
                if (m->sensitivity && m->n_sens > 0) {
                    for (uint32_t s = 0; s < m->n_sens; s++) {
                        const double sens = m->sensitivity[(size_t)i * m->n_sens + s];
                        if (fabs(sens) < 1e-16) continue;
                        double gx, gy, gz;
                        or_mot_gradient(density, g, px[i], py[i], pz[i], (int)s, layout, &gx, &gy, &gz);
                        bx += sens * gx;
                        by += sens * gy;
                        bz += sens * gz;
                    }
                } else {
                    double gx, gy, gz;
                    or_mot_gradient(density, g, px[i], py[i], pz[i], m->chemotaxis_index[i], layout, &gx, &gy, &gz);
                    const int dir = m->chemotaxis_direction[i];
                    bx = dir * gx;
                    by = dir * gy;
                    bz = dir * gz;
                }
                const double bmag = sqrt(bx * bx + by * by + bz * bz);
                if (bmag > 1e-16) {
                    bx /= bmag;
                    by /= bmag;
                    bz /= bmag;
                }
            }
            const double omb = 1.0 - bias;
            double mx = omb * rx + bias * bx;
            double my = omb * ry + bias * by;
            double mz = omb * rz + bias * bz;
            const double mag = sqrt(mx * mx + my * my + mz * mz);
            if (mag > 1e-16) {
                mx /= mag;
                my /= mag;
                mz /= mag;
            }
            const double sp = (double)speed[i];
            mvx[i] = mx * sp;
            mvy[i] = my * sp;
            mvz[i] = mz * sp;
        }
        vx[i] += (float)mvx[i];
        vy[i] += (float)mvy[i];
        vz[i] += (float)mvz[i];
    }
}

void or_run(const or_sim* sim, float* density, float* soa, uint32_t max_cells, uint32_t n_cells,
            const double* secretion, const double* uptake, const double* saturation,
            const double* net_export, const uint8_t* active,
            int n_diffusion_steps, double* mech_accum)
{
    or_run_motile(sim, density, soa, max_cells, n_cells, secretion, uptake, saturation, net_export, active,
                  n_diffusion_steps, mech_accum, NULL, 0, NULL, 0);
}

void or_run_motile(const or_sim* sim, float* density, float* soa, uint32_t max_cells, uint32_t n_cells,
                   const double* secretion, const double* uptake, const double* saturation,
                   const double* net_export, const uint8_t* active,
                   int n_diffusion_steps, double* mech_accum,
                   or_motility* mot, uint64_t seed, uint64_t* mot_step, int layout)
{
    const or_grid* g = &sim->grid;
    const or_mech* m = &sim->mech;
    const uint32_t V = m->mech_grid_nx * m->mech_grid_ny * m->mech_grid_nz;
    uint32_t* key = (uint32_t*)malloc(sizeof(uint32_t) * (n_cells ? n_cells : 1));
    uint32_t* order = (uint32_t*)malloc(sizeof(uint32_t) * (n_cells ? n_cells : 1));
    uint32_t* start = (uint32_t*)malloc(sizeof(uint32_t) * ((size_t)V + 1));
    const double dt_diff = (double)g->dt;
    const double dt_mech = (double)sim->dt_mechanics;
    for (int step = 0; step < n_diffusion_steps; step++) {
        or_diffusion_sweeps(density, g, sim->subs, OR_FP64);
        or_apply_dirichlet(density, g, sim->subs);
        if (n_cells) {
            const uint32_t* vox = (const uint32_t*)(soa + (size_t)OR_F_VOXEL_IDX * max_cells);
            const float* vol = soa + (size_t)OR_F_TOTAL_VOL * max_cells;
            or_secretion(density, g, n_cells, vox, vol, secretion, uptake, saturation,
                         net_export, active, dt_diff);
        }
        *mech_accum += dt_diff;
        if (*mech_accum >= dt_mech - 0.5 * dt_diff) {
            if (n_cells) {
                or_mech_bin(soa, max_cells, n_cells, m, g->x_min, g->y_min, g->z_min, key);
                or_mech_sort(key, n_cells, V, order, start);
                or_mech_forces(soa, max_cells, n_cells, m, key, order, start, NULL, NULL, NULL);
                if (mot) {
                    or_motility_update(soa, max_cells, n_cells, density, g, mot, dt_mech, seed, *mot_step, layout);
                    ++*mot_step;
                }
                or_mech_integrate_master(soa, max_cells, n_cells, m, g->x_min, g->y_min, g->z_min,
                                         (float)dt_mech, sim->pos64);
                if (sim->refresh_voxels) or_voxel_refresh(soa, max_cells, n_cells, g);
            }
            *mech_accum = 0.0;
        }
    }
    free(key); free(order); free(start);
}
