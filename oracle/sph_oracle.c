/*
 * sph_oracle.c — CPU restatement of the reference WCSPH step.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker for the CUDA path: only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 * The product library never links or calls it.
 *
 * It restates, in plain C (double precision for every field value, float for
 * the integer decisions that must match bit-exactly), the reference solver of
 * petbab/fluid-simulation:
 *
 *   Morton keys            src/cuda/nsearch/morton.cuh:7-34,
 *                          src/cuda/SPH/particle_data.cuh:117-125
 *   stable sort + gather   src/cuda/SPH/particle_data.cuh:112-133
 *   cell runs              src/cuda/tuning/kernels/rebuild_n_search.cu:10-36
 *   neighbour traversal    src/cuda/tuning/kernels/common.cuh:39-47,126-178
 *   SPH kernels            src/cuda/SPH/kernel.cuh:8-63
 *   density + Tait EOS     src/cuda/tuning/kernels/compute_rho_p.cu:87-100,223-225,301-316
 *   pressure + normals     src/cuda/tuning/kernels/compute_pressure_accel_n_normal.cu:99-123,346-364
 *   non-pressure accel     src/cuda/tuning/kernels/compute_non_pressure_accel.cu:114-144
 *   integrate + collisions src/cuda/tuning/kernels/update_positions.cu:14-68
 *   boundary masses        src/cuda/tuning/kernels/compute_boundary_mass.cu:10-30
 *   CFL time step          src/cuda/SPH/sph.cu:39-40,115-130
 *   state metrics          src/cuda/SPH/sph.cu:180-197
 *
 * Neighbour predicate: j != i and |x_i - x_j|^2 <= h^2 with the squared
 * distance rounded as fmaf(dz,dz,fmaf(dx,dx,dy*dy)) in float: the order nvcc
 * contracts the reference's dot(r, r) = x*x + y*y + z*z into (math.cuh:54-56),
 * which the CUDA path uses too, so neighbour sets compare bit-exactly.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/wcsph.h"

#ifdef _OPENMP
#include <omp.h>
#endif

typedef uint64_t u64;
typedef uint32_t u32;


/* ----------------------------------------------------------- Morton keys -- */
/* part_by_3 (morton.cuh:7-15) */
static u64 part_by_3(u64 n) {
    n &= 0x1fffffull;
    n = (n | (n << 32)) & 0x1f00000000ffffull;
    n = (n | (n << 16)) & 0x1f0000ff0000ffull;
    n = (n | (n << 8)) & 0x100f00f00f00f00full;
    n = (n | (n << 4)) & 0x10c30c30c30c30c3ull;
    n = (n | (n << 2)) & 0x1249249249249249ull;
    return n;
}
/* signed_to_unsigned (morton.cuh:18-21): + 2^20 with unsigned wrap */
static u32 offset_coord(int c) { return (u32)c + (1u << 20); }
/* encode_morton (morton.cuh:30-34) */
static u64 morton_of_cell(int cx, int cy, int cz) {
    return part_by_3(offset_coord(cx)) | (part_by_3(offset_coord(cy)) << 1) | (part_by_3(offset_coord(cz)) << 2);
}
/* key lambda (particle_data.cuh:117-125): floorf(p / cs) in float */
static void cell_of(const float* p, float cs, int* c) {
    c[0] = (int)floorf(p[0] / cs);
    c[1] = (int)floorf(p[1] / cs);
    c[2] = (int)floorf(p[2] / cs);
}

void oracle_morton_keys(const float* pos, u32 n, float cs, u64* keys) {
    for (u32 i = 0; i < n; ++i) {
        int c[3];
        cell_of(pos + 4 * (size_t)i, cs, c);
        keys[i] = morton_of_cell(c[0], c[1], c[2]);
    }
}

/* Stable LSD radix sort on 16-bit digits; perm[k] = input index of the k-th
 * smallest key (thrust::sort_by_key on (key, iota), particle_data.cuh:127). */
void oracle_sort_perm(const u64* keys, u32 n, u32* perm) {
    u32* a = perm;
    u32* b = (u32*)malloc(sizeof(u32) * (n ? n : 1));
    u32* cnt = (u32*)malloc(sizeof(u32) * 65537);
    for (u32 i = 0; i < n; ++i) a[i] = i;
    int swapped = 0;
    for (int pass = 0; pass < 4; ++pass) {
        const int sh = 16 * pass;
        memset(cnt, 0, sizeof(u32) * 65537);
        for (u32 i = 0; i < n; ++i) cnt[((keys[a[i]] >> sh) & 0xffffu) + 1]++;
        int trivial = 0;
        for (u32 d = 1; d <= 65536; ++d)
            if (cnt[d] == n) trivial = 1;
        if (trivial) continue;
        for (u32 d = 1; d <= 65536; ++d) cnt[d] += cnt[d - 1];
        for (u32 i = 0; i < n; ++i) b[cnt[(keys[a[i]] >> sh) & 0xffffu]++] = a[i];
        u32* t = a; a = b; b = t;
        swapped ^= 1;
    }
    if (swapped) { memcpy(b, a, sizeof(u32) * n); free(a); } else { free(b); }
    free(cnt);
}

/* ------------------------------------------------------------ cell index -- */
typedef struct {
    u32 ncells;
    u64* key;   /* Morton key of each cell, ascending */
    u32* start;
    u32* end;
} CellIndex;

/* Runs of equal cells in sorted order (rebuild_n_search.cu:19-34). */
static CellIndex build_cells(const float* spos, u32 n, float cs) {
    CellIndex ci;
    ci.ncells = 0;
    ci.key = (u64*)malloc(sizeof(u64) * (n ? n : 1));
    ci.start = (u32*)malloc(sizeof(u32) * (n ? n : 1));
    ci.end = (u32*)malloc(sizeof(u32) * (n ? n : 1));
    u64 prev = 0;
    for (u32 i = 0; i < n; ++i) {
        int c[3];
        cell_of(spos + 4 * (size_t)i, cs, c);
        const u64 k = morton_of_cell(c[0], c[1], c[2]);
        if (i == 0 || k != prev) {
            if (i) ci.end[ci.ncells - 1] = i;
            ci.key[ci.ncells] = k;
            ci.start[ci.ncells] = i;
            ci.ncells++;
        }
        prev = k;
    }
    if (n) ci.end[ci.ncells - 1] = n;
    return ci;
}
static void free_cells(CellIndex* ci) { free(ci->key); free(ci->start); free(ci->end); }

static int find_cell(const CellIndex* ci, u64 key, u32* s, u32* e) {
    u32 lo = 0, hi = ci->ncells;
    while (lo < hi) {
        const u32 mid = (lo + hi) >> 1;
        if (ci->key[mid] < key) lo = mid + 1; else hi = mid;
    }
    if (lo < ci->ncells && ci->key[lo] == key) { *s = ci->start[lo]; *e = ci->end[lo]; return 1; }
    return 0;
}

/* Exported: cell runs as (morton key, start, end) for parity of cell ranges. */
u32 oracle_cell_ranges(const float* spos, u32 n, float cs, u64* keys_out, u32* start_out, u32* end_out) {
    CellIndex ci = build_cells(spos, n, cs);
    const u32 nc = ci.ncells;
    if (keys_out) memcpy(keys_out, ci.key, sizeof(u64) * nc);
    if (start_out) memcpy(start_out, ci.start, sizeof(u32) * nc);
    if (end_out) memcpy(end_out, ci.end, sizeof(u32) * nc);
    free_cells(&ci);
    return nc;
}

/* ---------------------------------------------------------- SPH formulas -- */
static float dist2f(const float* a, const float* b) {
    const float dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    return fmaf(dz, dz, fmaf(dx, dx, dy * dy));
}

typedef struct {
    double r, spacing, h, mass, rho0, k, gamma, max_ratio, nu, alpha, g[3];
    double cubic_f, cubic_grad_f, spiky_grad_f, cohesion_f, visc_eps;
    float hf, h2f, csf, bufferf, rf, spacingf;
    int R;
} Consts;

static Consts make_consts(const wcsph_params* P) {
    Consts c;
    c.rf = P->particle_radius;
    c.spacingf = 2.f * c.rf;
    c.hf = 2.f * c.spacingf;
    c.h2f = c.hf * c.hf;
    c.csf = c.hf * P->cell_size_mult;
    c.bufferf = c.rf * P->collision_buffer_mult;
    c.r = c.rf;
    c.spacing = c.spacingf;
    c.h = c.hf;
    c.mass = (double)P->rest_density * (c.spacing * c.spacing * c.spacing * 0.8);
    c.rho0 = P->rest_density;
    c.k = P->stiffness;
    c.gamma = P->exponent;
    c.max_ratio = P->max_density_ratio;
    c.nu = P->viscosity;
    c.alpha = P->surface_tension;
    for (int d = 0; d < 3; ++d) c.g[d] = P->gravity[d];
    const double pi = 3.14159265358979323846;
    c.cubic_f = 8.0 / (pi * c.h * c.h * c.h);
    c.cubic_grad_f = 48.0 / (pi * c.h * c.h * c.h);
    c.spiky_grad_f = -45.0 / (pi * pow(c.h, 9.0));
    c.cohesion_f = 32.0 / (pi * c.h * c.h * c.h);
    c.visc_eps = 0.01 * c.h * c.h;
    c.R = (int)(c.hf / c.csf + .5f); /* common.cuh:131 */
    return c;
}

/* cubic_spline (kernel.cuh:12-19) */
static double cubic_w(double q, const Consts* c) {
    if (q <= 0.5) return c->cubic_f * (6.0 * q * q * q - 6.0 * q * q + 1.0);
    if (q <= 1.0) return c->cubic_f * 2.0 * (1.0 - q) * (1.0 - q) * (1.0 - q);
    return 0.0;
}
/* cubic_spline_grad (kernel.cuh:22-32), coefficient of r */
static double cubic_grad(double q, const Consts* c) {
    if (q < 1e-9 || q > 1.0) return 0.0;
    const double rl = q * c->h;
    if (q <= 0.5) return c->cubic_grad_f * q * (3.0 * q - 2.0) / (c->h * rl);
    return -c->cubic_grad_f * (1.0 - q) * (1.0 - q) / (c->h * rl);
}
/* spiky_grad (kernel.cuh:43-51), coefficient of r */
static double spiky_grad(double q, const Consts* c) {
    if (q < 1e-9 || q > 1.0) return 0.0;
    const double rl = q * c->h;
    return c->spiky_grad_f * (1.0 - q) * (1.0 - q) / (c->h * rl);
}
/* cohesion (kernel.cuh:53-63) */
static double cohesion(double q, const Consts* c) {
    const double iq3 = (1.0 - q) * (1.0 - q) * (1.0 - q), q3 = q * q * q;
    if (q <= 0.5) return c->cohesion_f * (2.0 * q3 * iq3 - 1.0 / 64.0);
    if (q <= 1.0) return c->cohesion_f * q3 * iq3;
    return 0.0;
}

static void external_force(const wcsph_params* P, const double* x, double* f) {
    f[0] = f[1] = f[2] = 0.0;
    switch (P->external_force) {
    case WCSPH_FORCE_CONSTANT:
        f[0] = P->external_force_param[0]; f[1] = P->external_force_param[1]; f[2] = P->external_force_param[2];
        break;
    case WCSPH_FORCE_FOUNTAIN: /* app/fountain/application.cu:36-42 */
        if (x[0] * x[0] + x[2] * x[2] < .2 && x[1] < 0.0) { f[1] = 25.0; break; }
        if (x[1] < -0.3) {
            const double l = sqrt(x[0] * x[0] + x[2] * x[2]);
            f[0] = 2.0 * (-x[0] / l); f[2] = 2.0 * (-x[2] / l);
        }
        break;
    case WCSPH_FORCE_VORTEX: /* app/vortex/application.cu:45 */
        if (x[1] < -0.5) {
            const double l = sqrt(x[2] * x[2] + x[0] * x[0]);
            f[0] = 2.0 * (x[2] / l); f[2] = 2.0 * (-x[0] / l);
        }
        break;
    default: break;
    }
}

/* mat4 * float4 (math.cuh:78-86), column-major */
static void mat_mul(const float* m, const double* v, double* out) {
    for (int r = 0; r < 4; ++r)
        out[r] = m[r] * v[0] + m[4 + r] * v[1] + m[8 + r] * v[2] + m[12 + r] * v[3];
}

/* -------------------------------------------------- boundary preparation -- */
/* Boundary sort (particle_data.cuh:84-110) with cell = h and masses
 * m_b = rho0 / (W(0) + sum_b' W) (compute_boundary_mass.cu:10-30). */
void oracle_boundary_init(const wcsph_params* P, u32 nb, const float* bpos_in, float* bpos_sorted, double* bmass) {
    Consts c = make_consts(P);
    u64* keys = (u64*)malloc(sizeof(u64) * (nb ? nb : 1));
    u32* perm = (u32*)malloc(sizeof(u32) * (nb ? nb : 1));
    oracle_morton_keys(bpos_in, nb, c.hf, keys);
    oracle_sort_perm(keys, nb, perm);
    for (u32 i = 0; i < nb; ++i) memcpy(bpos_sorted + 4 * (size_t)i, bpos_in + 4 * (size_t)perm[i], 16);
    CellIndex ci = build_cells(bpos_sorted, nb, c.hf);
#pragma omp parallel for schedule(dynamic, 256)
    for (long long ii = 0; ii < (long long)nb; ++ii) {
        const u32 i = (u32)ii;
        const float* xi = bpos_sorted + 4 * (size_t)i;
        int cc[3];
        cell_of(xi, c.hf, cc);
        double sum = cubic_w(0.0, &c);
        for (int x = -1; x <= 1; ++x)
            for (int y = -1; y <= 1; ++y)
                for (int z = -1; z <= 1; ++z) {
                    u32 s, e;
                    if (!find_cell(&ci, morton_of_cell(cc[0] + x, cc[1] + y, cc[2] + z), &s, &e)) continue;
                    for (u32 j = s; j < e; ++j) {
                        const float* xj = bpos_sorted + 4 * (size_t)j;
                        if (j == i || dist2f(xi, xj) > c.h2f) continue;
                        const double dx = (double)xi[0] - xj[0], dy = (double)xi[1] - xj[1], dz = (double)xi[2] - xj[2];
                        sum += cubic_w(sqrt(dx * dx + dy * dy + dz * dz) / c.h, &c);
                    }
                }
        bmass[i] = c.rho0 / sum;
    }
    free_cells(&ci);
    free(keys);
    free(perm);
}

/* ------------------------------------------------------------- one step -- */
typedef struct {
    u32* cnt;
    u32* off;
    u32* idx;
    u64 total;
} Csr;

/* Fluid neighbour lists in the reference traversal order (for_neighbors,
 * common.cuh:126-151: x, y, z nested; ascending j inside a cell). */
static Csr build_neighbors(const float* spos, u32 n, const Consts* c, const CellIndex* ci) {
    Csr L;
    L.cnt = (u32*)calloc(n ? n : 1, sizeof(u32));
    L.off = (u32*)calloc(n ? n : 1, sizeof(u32));
    const int R = c->R;
#pragma omp parallel for schedule(dynamic, 256)
    for (long long ii = 0; ii < (long long)n; ++ii) {
        const u32 i = (u32)ii;
        const float* xi = spos + 4 * (size_t)i;
        int cc[3];
        cell_of(xi, c->csf, cc);
        u32 k = 0;
        for (int x = -R; x <= R; ++x)
            for (int y = -R; y <= R; ++y)
                for (int z = -R; z <= R; ++z) {
                    u32 s, e;
                    if (!find_cell(ci, morton_of_cell(cc[0] + x, cc[1] + y, cc[2] + z), &s, &e)) continue;
                    for (u32 j = s; j < e; ++j)
                        if (j != i && dist2f(xi, spos + 4 * (size_t)j) <= c->h2f) ++k;
                }
        L.cnt[i] = k;
    }
    u64 run = 0;
    for (u32 i = 0; i < n; ++i) { L.off[i] = (u32)run; run += L.cnt[i]; }
    L.total = run;
    L.idx = (u32*)malloc(sizeof(u32) * (run ? run : 1));
#pragma omp parallel for schedule(dynamic, 256)
    for (long long ii = 0; ii < (long long)n; ++ii) {
        const u32 i = (u32)ii;
        const float* xi = spos + 4 * (size_t)i;
        int cc[3];
        cell_of(xi, c->csf, cc);
        u32 w = L.off[i];
        for (int x = -R; x <= R; ++x)
            for (int y = -R; y <= R; ++y)
                for (int z = -R; z <= R; ++z) {
                    u32 s, e;
                    if (!find_cell(ci, morton_of_cell(cc[0] + x, cc[1] + y, cc[2] + z), &s, &e)) continue;
                    for (u32 j = s; j < e; ++j)
                        if (j != i && dist2f(xi, spos + 4 * (size_t)j) <= c->h2f) L.idx[w++] = j;
                }
    }
    return L;
}

/* Everything one step computes, in sorted particle order. */
typedef struct {
    u64* keys;      /* [n] input order */
    u32* perm;      /* [n] sorted -> input index */
    double* rho;    /* [n] */
    double* prs;    /* [n] */
    double* ap;     /* [4n] */
    double* anp;    /* [4n] */
    double* normal; /* [4n] */
    double* pos;    /* [4n] state after the step */
    double* vel;    /* [4n] */
    double dt_p, np_dt;
    u32* nbr_cnt;   /* [n] */
    u32* nbr_off;   /* [n] */
    u32* nbr_idx;   /* [cap] */
    u64 nbr_cap;
    u64 nbr_total;
} OracleOut;

/* adapt_time_step (sph.cu:115-130) in float, as the reference host code. */
static float adapt_time_step(const wcsph_params* P, const float* vel, u32 n, float delta) {
    float vmax2 = 0.f;
    for (u32 i = 0; i < n; ++i) {
        const float* v = vel + 4 * (size_t)i;
        const float s = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        if (s > vmax2) vmax2 = s;
    }
    const float vmax = sqrtf(vmax2);
    const float lo = P->min_time_step, hi = P->max_time_step;
    const float clamped = delta < lo ? lo : (hi < delta ? hi : delta);
    if (P->cfl_factor <= 0.f) return clamped;
    if ((double)vmax < 1.e-9) return hi;
    const float spacing = 2.f * P->particle_radius;
    const float cfl = (P->cfl_factor * spacing) / vmax;
    return cfl < clamped ? cfl : clamped;
}

/* One FluidSimulator::update(delta) of CUDASPHSimulator (sph.cu:31-60). */
int oracle_step(const wcsph_params* P, const wcsph_box* box, u32 n, const float* pos_in, const float* vel_in,
                u32 nb, const float* bpos, const double* bmass, float delta, OracleOut* out) {
    Consts c = make_consts(P);
    const float np_dt_f = delta < P->non_pressure_max_time_step ? delta : P->non_pressure_max_time_step;
    const float dt_f = adapt_time_step(P, vel_in, n, delta);
    out->dt_p = dt_f;
    out->np_dt = np_dt_f;
    const double dt = dt_f, np_dt = np_dt_f;

    /* sort (particle_data.cuh:112-133) */
    oracle_morton_keys(pos_in, n, c.csf, out->keys);
    oracle_sort_perm(out->keys, n, out->perm);
    float* spos = (float*)malloc(sizeof(float) * 4 * (n ? n : 1));
    float* svel = (float*)malloc(sizeof(float) * 4 * (n ? n : 1));
    for (u32 i = 0; i < n; ++i) {
        memcpy(spos + 4 * (size_t)i, pos_in + 4 * (size_t)out->perm[i], 16);
        memcpy(svel + 4 * (size_t)i, vel_in + 4 * (size_t)out->perm[i], 16);
    }
    CellIndex ci = build_cells(spos, n, c.csf);
    CellIndex bci;
    memset(&bci, 0, sizeof(bci));
    if (nb) bci = build_cells(bpos, nb, c.hf);
    Csr L = build_neighbors(spos, n, &c, &ci);
    out->nbr_total = L.total;

    double* vlap = (double*)calloc(4 * (size_t)(n ? n : 1), sizeof(double));

    /* density + EOS (compute_rho_p.cu:87-100 + boundary :301-316) */
#pragma omp parallel for schedule(dynamic, 256)
    for (long long ii = 0; ii < (long long)n; ++ii) {
        const u32 i = (u32)ii;
        const float* xi = spos + 4 * (size_t)i;
        double w = cubic_w(0.0, &c);
        for (u32 k = L.off[i]; k < L.off[i] + L.cnt[i]; ++k) {
            const float* xj = spos + 4 * (size_t)L.idx[k];
            const double dx = (double)xi[0] - xj[0], dy = (double)xi[1] - xj[1], dz = (double)xi[2] - xj[2];
            w += cubic_w(sqrt(dx * dx + dy * dy + dz * dz) / c.h, &c);
        }
        double rho = w * c.mass;
        if (nb) {
            int bc[3];
            cell_of(xi, c.hf, bc);
            for (int x = -1; x <= 1; ++x)
                for (int y = -1; y <= 1; ++y)
                    for (int z = -1; z <= 1; ++z) {
                        u32 s, e;
                        if (!find_cell(&bci, morton_of_cell(bc[0] + x, bc[1] + y, bc[2] + z), &s, &e)) continue;
                        for (u32 b = s; b < e; ++b) {
                            const float* xb = bpos + 4 * (size_t)b;
                            if (dist2f(xi, xb) > c.h2f) continue;
                            const double dx = (double)xi[0] - xb[0], dy = (double)xi[1] - xb[1],
                                         dz = (double)xi[2] - xb[2];
                            rho += cubic_w(sqrt(dx * dx + dy * dy + dz * dz) / c.h, &c) * bmass[b];
                        }
                    }
        }
        out->rho[i] = rho;
        double ratio = rho / c.rho0;
        if (ratio < 1.0) ratio = 1.0;
        if (ratio > c.max_ratio) ratio = c.max_ratio;
        out->prs[i] = c.k * (pow(ratio, c.gamma) - 1.0);
    }

    /* pressure accel + normals (compute_pressure_accel_n_normal.cu:99-123,
     * boundary :346-364) and the viscosity Laplacian
     * (compute_non_pressure_accel.cu:138-140) */
#pragma omp parallel for schedule(dynamic, 256)
    for (long long ii = 0; ii < (long long)n; ++ii) {
        const u32 i = (u32)ii;
        const float* xi = spos + 4 * (size_t)i;
        const float* vi = svel + 4 * (size_t)i;
        const double di = out->rho[i], pi = out->prs[i];
        const double dpi = pi / (di * di);
        double a[3] = {0, 0, 0}, nr[3] = {0, 0, 0}, vl[3] = {0, 0, 0};
        for (u32 k = L.off[i]; k < L.off[i] + L.cnt[i]; ++k) {
            const u32 j = L.idx[k];
            const float* xj = spos + 4 * (size_t)j;
            const float* vj = svel + 4 * (size_t)j;
            const double r[3] = {(double)xi[0] - xj[0], (double)xi[1] - xj[1], (double)xi[2] - xj[2]};
            const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
            const double q = sqrt(r2) / c.h;
            const double dj = out->rho[j], pj = out->prs[j];
            const double sg = spiky_grad(q, &c), cg = cubic_grad(q, &c);
            const double coef = (dpi + pj / (dj * dj)) * sg;
            const double vr = ((double)vi[0] - vj[0]) * r[0] + ((double)vi[1] - vj[1]) * r[1] +
                              ((double)vi[2] - vj[2]) * r[2];
            const double s = vr * cg / (dj * (r2 + c.visc_eps));
            for (int d = 0; d < 3; ++d) {
                a[d] -= coef * r[d];
                nr[d] += r[d] * cg / dj;
                vl[d] += s * r[d];
            }
        }
        for (int d = 0; d < 3; ++d) a[d] *= c.mass;
        if (nb) {
            const double b_p_term = dpi + pi / (c.rho0 * c.rho0);
            int bc[3];
            cell_of(xi, c.hf, bc);
            for (int x = -1; x <= 1; ++x)
                for (int y = -1; y <= 1; ++y)
                    for (int z = -1; z <= 1; ++z) {
                        u32 s, e;
                        if (!find_cell(&bci, morton_of_cell(bc[0] + x, bc[1] + y, bc[2] + z), &s, &e)) continue;
                        for (u32 b = s; b < e; ++b) {
                            const float* xb = bpos + 4 * (size_t)b;
                            if (dist2f(xi, xb) > c.h2f) continue;
                            const double r[3] = {(double)xi[0] - xb[0], (double)xi[1] - xb[1], (double)xi[2] - xb[2]};
                            const double q = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]) / c.h;
                            const double coef = bmass[b] * b_p_term * spiky_grad(q, &c);
                            for (int d = 0; d < 3; ++d) a[d] -= coef * r[d];
                        }
                    }
        }
        for (int d = 0; d < 3; ++d) {
            out->ap[4 * (size_t)i + d] = a[d];
            out->normal[4 * (size_t)i + d] = c.h * c.mass * nr[d];
            vlap[4 * (size_t)i + d] = vl[d];
        }
        out->ap[4 * (size_t)i + 3] = 0.0;
        out->normal[4 * (size_t)i + 3] = 0.0;
    }

    /* surface tension + non-pressure accel (compute_non_pressure_accel.cu:114-144),
     * then integrate + box collision (update_positions.cu:54-68) */
#pragma omp parallel for schedule(dynamic, 256)
    for (long long ii = 0; ii < (long long)n; ++ii) {
        const u32 i = (u32)ii;
        const float* xi = spos + 4 * (size_t)i;
        const double di = out->rho[i];
        const double* ni = out->normal + 4 * (size_t)i;
        double f[3] = {0, 0, 0};
        for (u32 k = L.off[i]; k < L.off[i] + L.cnt[i]; ++k) {
            const u32 j = L.idx[k];
            const float* xj = spos + 4 * (size_t)j;
            const double r[3] = {(double)xi[0] - xj[0], (double)xi[1] - xj[1], (double)xi[2] - xj[2]};
            const double r2f = (double)dist2f(xi, xj);
            if (!(r2f > 1e-6)) continue;
            const double len = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
            const double q = len / c.h;
            const double C = cohesion(q, &c);
            const double dj = out->rho[j];
            const double* nj = out->normal + 4 * (size_t)j;
            for (int d = 0; d < 3; ++d) f[d] += (c.mass * (r[d] / len) * C + ni[d] - nj[d]) / (di + dj);
        }
        double xd[4] = {xi[0], xi[1], xi[2], xi[3]};
        double fe[3];
        external_force(P, xd, fe);
        double anp[3];
        for (int d = 0; d < 3; ++d)
            anp[d] = c.g[d] + fe[d] + c.nu * 10.0 * c.mass * vlap[4 * (size_t)i + d] - c.alpha * 2.0 * c.rho0 * f[d];
        for (int d = 0; d < 3; ++d) out->anp[4 * (size_t)i + d] = anp[d];
        out->anp[4 * (size_t)i + 3] = 0.0;
        const float* vi = svel + 4 * (size_t)i;
        double v[4] = {vi[0], vi[1], vi[2], vi[3]};
        for (int d = 0; d < 3; ++d) v[d] += np_dt * anp[d] + dt * out->ap[4 * (size_t)i + d];
        double x[4];
        for (int d = 0; d < 4; ++d) x[d] = xd[d] + dt * v[d];
        /* resolve_collisions (update_positions.cu:14-52) */
        double p[4], u[4];
        mat_mul(box->model_inv, x, p);
        mat_mul(box->model_inv, v, u);
        int changed = 0;
        const double buf = c.bufferf, rr = c.rf, el = P->elasticity;
        for (int d = 0; d < 3; ++d) {
            if (p[d] - buf < box->min[d]) { p[d] = (double)box->min[d] + rr; u[d] *= -el; changed = 1; }
            else if (p[d] + buf > box->max[d]) { p[d] = (double)box->max[d] - rr; u[d] *= -el; changed = 1; }
        }
        if (changed) {
            mat_mul(box->model, p, x);
            mat_mul(box->model, u, v);
        }
        for (int d = 0; d < 4; ++d) {
            out->pos[4 * (size_t)i + d] = x[d];
            out->vel[4 * (size_t)i + d] = v[d];
        }
    }

    if (out->nbr_cnt) memcpy(out->nbr_cnt, L.cnt, sizeof(u32) * n);
    if (out->nbr_off) memcpy(out->nbr_off, L.off, sizeof(u32) * n);
    if (out->nbr_idx && L.total <= out->nbr_cap) memcpy(out->nbr_idx, L.idx, sizeof(u32) * L.total);

    free(vlap);
    free(L.cnt); free(L.off); free(L.idx);
    free_cells(&ci);
    if (nb) free_cells(&bci);
    free(spos);
    free(svel);
    return 0;
}

/* Flat-argument wrapper for ctypes callers. */
int oracle_step_flat(const wcsph_params* P, const wcsph_box* box, u32 n, const float* pos_in, const float* vel_in,
                     u32 nb, const float* bpos, const double* bmass, float delta, u64* keys, u32* perm, double* rho,
                     double* prs, double* ap, double* anp, double* normal, double* pos_out, double* vel_out,
                     double* dt_out, u32* nbr_cnt, u32* nbr_off, u32* nbr_idx, u64 nbr_cap, u64* nbr_total) {
    OracleOut o;
    o.keys = keys; o.perm = perm; o.rho = rho; o.prs = prs; o.ap = ap; o.anp = anp; o.normal = normal;
    o.pos = pos_out; o.vel = vel_out; o.nbr_cnt = nbr_cnt; o.nbr_off = nbr_off; o.nbr_idx = nbr_idx;
    o.nbr_cap = nbr_cap; o.nbr_total = 0;
    const int s = oracle_step(P, box, n, pos_in, vel_in, nb, bpos, bmass, delta, &o);
    if (dt_out) { dt_out[0] = o.dt_p; dt_out[1] = o.np_dt; }
    if (nbr_total) *nbr_total = o.nbr_total;
    return s;
}

/* mean_speed = sum|v|/N, ke = sum 0.5 m |v|^2 (sph.cu:180-197) */
void oracle_metrics(const wcsph_params* P, u32 n, const float* vel, double* mean_speed, double* ke) {
    const float s = 2.f * P->particle_radius;
    const double mass = (double)P->rest_density * (float)((double)(s * s * s) * 0.8);
    double a = 0, b = 0;
    for (u32 i = 0; i < n; ++i) {
        const float* v = vel + 4 * (size_t)i;
        const double d = (double)v[0] * v[0] + (double)v[1] * v[1] + (double)v[2] * v[2];
        a += sqrt(d);
        b += 0.5 * mass * d;
    }
    *mean_speed = n ? a / n : 0.0;
    *ke = b;
}

int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
