/*
 * mpcd_oracle.c — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C CPU restatement of the reference SRC/MPCD time step
 * (llemoyne1/SRC_incompressible_openMP). It is the checker for the CUDA path: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg may load it. The product library
 * never links or calls it.
 *
 * Pinning: tests/test_oracle_vs_reference.py runs this oracle and the unmodified reference
 * (built from its own sources by oracle/Makefile into oracle/_ref/) on the same seeded inputs
 * and requires bit-identical outputs for every phase; tests/golden/ holds fixtures produced
 * by the reference for the cases that run without it.
 *
 * Every function cites the reference file:line it restates. The RNG follows libstdc++ 13
 * (GCC 13.3): std::mt19937_64 (Matsumoto-Nishimura MT19937-64), generate_canonical<double,53>,
 * uniform_int_distribution (Lemire's nearly-divisionless method on 128-bit products),
 * normal_distribution (Marsaglia polar method with one cached deviate) and std::shuffle
 * (Fisher-Yates drawing two swap positions per call when the range allows). Those are
 * restated from the published algorithms; the reference's call sites are cited at each use.
 *
 * Zone passes are restated zone-locally: a zone's kernel reads only the snapshot's cell
 * counts (its rectangle plus a 2-cell halo) and the particle lists of its own cells, and
 * moves particles only between its own cells, so it never needs the reference's O(n) full
 * copy per zone (src/zone_pass_openmp.cpp:67-72). Results are identical.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mpcd_c.h"

typedef mpcd_params_c P;

static char g_err[512];
const char* oracle_last_error(void) { return g_err; }
static int fail(int code, const char* msg) {
    snprintf(g_err, sizeof g_err, "%s", msg);
    return code;
}

/* ======================================================================== RNG */

typedef struct {
    uint64_t s[312];
    int i;
} mt64;

static void mt_seed(mt64* r, uint64_t seed) {
    r->s[0] = seed;
    for (int i = 1; i < 312; ++i) r->s[i] = 6364136223846793005ULL * (r->s[i - 1] ^ (r->s[i - 1] >> 62)) + (uint64_t)i;
    r->i = 312;
}

static void mt_twist(mt64* r) {
    const uint64_t UM = 0xFFFFFFFF80000000ULL, LM = 0x7FFFFFFFULL;
    for (int k = 0; k < 312; ++k) {
        const uint64_t y = (r->s[k] & UM) | (r->s[(k + 1) % 312] & LM);
        r->s[k] = r->s[(k + 156) % 312] ^ (y >> 1) ^ ((y & 1ULL) ? 0xB5026F5AA96619E9ULL : 0ULL);
    }
    r->i = 0;
}

static uint64_t mt_next(mt64* r) {
    if (r->i >= 312) mt_twist(r);
    uint64_t z = r->s[r->i++];
    z ^= (z >> 29) & 0x5555555555555555ULL;
    z ^= (z << 17) & 0x71D67FFFEDA60000ULL;
    z ^= (z << 37) & 0xFFF7EEE000000000ULL;
    z ^= z >> 43;
    return z;
}

/* generate_canonical<double, 53> with a 64-bit engine: one draw, u / 2^64, kept below 1 */
static double canon(mt64* r) {
    double c = (double)mt_next(r) / 18446744073709551616.0;
    if (c >= 1.0) c = nextafter(1.0, 0.0);
    return c;
}

/* uniform_real_distribution<double>(a, b): canonical * (b - a) + a */
static double unif(mt64* r, double a, double b) { return canon(r) * (b - a) + a; }

/* uniform_int_distribution on [lo, hi] with a 64-bit engine (Lemire downscaling) */
static uint64_t unif_int(mt64* r, uint64_t lo, uint64_t hi) {
    const uint64_t range = hi - lo + 1ULL;
    unsigned __int128 prod = (unsigned __int128)mt_next(r) * range;
    uint64_t low = (uint64_t)prod;
    if (low < range) {
        const uint64_t thr = (0ULL - range) % range;
        while (low < thr) {
            prod = (unsigned __int128)mt_next(r) * range;
            low = (uint64_t)prod;
        }
    }
    return (uint64_t)(prod >> 64) + lo;
}

/* normal_distribution<double>(0, 1): Marsaglia polar method, one cached deviate */
typedef struct {
    double saved;
    int has;
} normal_st;

static double normal01(normal_st* nd, mt64* r) {
    double ret;
    if (nd->has) {
        nd->has = 0;
        ret = nd->saved;
    } else {
        double x, y, r2;
        do {
            x = 2.0 * canon(r) - 1.0;
            y = 2.0 * canon(r) - 1.0;
            r2 = x * x + y * y;
        } while (r2 > 1.0 || r2 == 0.0);
        const double mult = sqrt(-2.0 * log(r2) / r2);
        nd->saved = x * mult;
        nd->has = 1;
        ret = y * mult;
    }
    return ret * 1.0 + 0.0;
}

/* std::shuffle of n ints (the two-positions-per-draw branch; n is always far below 2^32) */
static void shuffle_ints(int* a, int n, mt64* r) {
    if (n <= 0) return;
    int i = 1;
    if ((n % 2) == 0) {
        const int j = (int)unif_int(r, 0, 1);
        const int t = a[i]; a[i] = a[j]; a[j] = t;
        ++i;
    }
    while (i != n) {
        const uint64_t sr = (uint64_t)i + 1ULL;
        const uint64_t x = unif_int(r, 0, sr * (sr + 1ULL) - 1ULL);
        const int p1 = (int)(x / (sr + 1ULL)), p2 = (int)(x % (sr + 1ULL));
        int t = a[i]; a[i] = a[p1]; a[p1] = t;
        ++i;
        t = a[i]; a[i] = a[p2]; a[p2] = t;
        ++i;
    }
}

/* KAT entry points for tests (draw sequences compared with libstdc++) */
void oracle_rng_kat(uint64_t seed, int kind, int count, double* out, uint64_t* outu) {
    mt64 r;
    mt_seed(&r, seed);
    normal_st nd = {0.0, 0};
    for (int k = 0; k < count; ++k) {
        if (kind == 0) outu[k] = mt_next(&r);
        else if (kind == 1) out[k] = canon(&r);
        else if (kind == 2) out[k] = normal01(&nd, &r);
        else if (kind == 3) outu[k] = unif_int(&r, 1, 8);
        else if (kind == 4) outu[k] = unif_int(&r, 0, (uint64_t)(k % 37) + 1ULL);
    }
}

void oracle_shuffle_kat(uint64_t seed, int n, int* a) {
    mt64 r;
    mt_seed(&r, seed);
    shuffle_ints(a, n, &r);
}

/* ================================================================ grid helpers */

static double dmax(double a, double b) { return (a < b) ? b : a; } /* std::max semantics */
static double dmin(double a, double b) { return (b < a) ? b : a; } /* std::min semantics */
static int imax(int a, int b) { return (a < b) ? b : a; }
static int imin(int a, int b) { return (b < a) ? b : a; }
static int periodic_x(const P* p) { return p->boundary_left == MPCD_BC_PERIODIC && p->boundary_right == MPCD_BC_PERIODIC; }
static int periodic_y(const P* p) { return p->boundary_bottom == MPCD_BC_PERIODIC && p->boundary_top == MPCD_BC_PERIODIC; }
static int wrap_index(int i, int n) { int r = i % n; return (r < 0) ? r + n : r; }

/* src/common_grid.cpp:9-19 */
static int cell_of(double x, double y, const P* p) {
    const double dx = p->Lx / (double)p->Nx, dy = p->Ly / (double)p->Ny;
    int ix = (int)floor(x / dx), iy = (int)floor(y / dy);
    if (ix < 0) ix = 0;
    if (ix >= p->Nx) ix = p->Nx - 1;
    if (iy < 0) iy = 0;
    if (iy >= p->Ny) iy = p->Ny - 1;
    return iy + p->Ny * ix;
}

void oracle_cell_ids(const P* p, const double* x, int32_t* cid) {
    for (int i = 0; i < p->n; ++i) cid[i] = cell_of(x[2 * i], x[2 * i + 1], p);
}

/* ================================================================== stream + BC */

/* src/main_benchmark_poiseuille_openmp_profiled_shifted_profiled.cpp:242-247 */
void oracle_stream(const P* p, double* x, double* v) {
    for (int i = 0; i < p->n; ++i) {
        v[2 * i] += p->bodyForceX * p->dt;
        v[2 * i + 1] += p->g * p->dt;
        x[2 * i] += p->dt * v[2 * i];
        x[2 * i + 1] += p->dt * v[2 * i + 1];
    }
}

static const char* bc_side_name(int side) {
    static const char* names[4] = {"boundary_left", "boundary_right", "boundary_bottom", "boundary_top"};
    return names[side];
}

/* src/boundary_conditions.cpp:19-203 */
int oracle_apply_bc(const P* p, double* x, double* v, uint64_t seed, mpcd_wallinfo_c* info) {
    mt64 r;
    mt_seed(&r, seed);
    normal_st nd = {0.0, 0};
    mpcd_wallinfo_c w;
    memset(&w, 0, sizeof w);
    const double Lx = p->Lx, Ly = p->Ly, sig = p->wallSigma;
    for (int k = 0; k < 4; ++k) {
        for (int i = 0; i < p->n; ++i) {
            double* xi = &x[2 * i];
            double* yi = &x[2 * i + 1];
            double* vx = &v[2 * i];
            double* vy = &v[2 * i + 1];
            if (*xi < 0.0) {
                const double ox = *vx, oy = *vy;
                const int m = p->boundary_left;
                if (m == MPCD_BC_PERIODIC) {
                    *xi += Lx;
                } else if (m == MPCD_BC_THERMALIZE || m == MPCD_BC_BOUNCEBACK || m == MPCD_BC_SPECULAR) {
                    *xi = -*xi;
                    if (m == MPCD_BC_THERMALIZE) {
                        *vx = fabs(sig * normal01(&nd, &r));
                        *vy = sig * normal01(&nd, &r);
                    } else if (m == MPCD_BC_BOUNCEBACK) {
                        *vx = fabs(*vx);
                        *vy = -*vy;
                    } else {
                        *vx = fabs(*vx);
                    }
                    const double dvx = *vx - ox, dvy = *vy - oy;
                    w.nLeft += 1;
                    w.dEwall += 0.5 * ((*vx * *vx + *vy * *vy) - (ox * ox + oy * oy));
                    w.dPxLeft += fabs(dvx);
                    w.dPyLeft += dvy;
                } else {
                    return fail(MPCD_ERR_UNSUPPORTED_BC, "Unsupported boundary_left mode");
                }
            }
            if (*xi > Lx) {
                const double ox = *vx, oy = *vy;
                const int m = p->boundary_right;
                if (m == MPCD_BC_PERIODIC) {
                    *xi -= Lx;
                } else if (m == MPCD_BC_THERMALIZE || m == MPCD_BC_BOUNCEBACK || m == MPCD_BC_SPECULAR) {
                    *xi = 2.0 * Lx - *xi;
                    if (m == MPCD_BC_THERMALIZE) {
                        *vx = -fabs(sig * normal01(&nd, &r));
                        *vy = sig * normal01(&nd, &r);
                    } else if (m == MPCD_BC_BOUNCEBACK) {
                        *vx = -fabs(*vx);
                        *vy = -*vy;
                    } else {
                        *vx = -fabs(*vx);
                    }
                    const double dvx = *vx - ox, dvy = *vy - oy;
                    w.nRight += 1;
                    w.dEwall += 0.5 * ((*vx * *vx + *vy * *vy) - (ox * ox + oy * oy));
                    w.dPxRight += fabs(dvx);
                    w.dPyRight += dvy;
                } else {
                    return fail(MPCD_ERR_UNSUPPORTED_BC, "Unsupported boundary_right mode");
                }
            }
            if (*yi < 0.0) {
                const double ox = *vx, oy = *vy;
                const int m = p->boundary_bottom;
                if (m == MPCD_BC_PERIODIC) {
                    *yi += Ly;
                } else if (m == MPCD_BC_THERMALIZE || m == MPCD_BC_BOUNCEBACK || m == MPCD_BC_SPECULAR) {
                    *yi = -*yi;
                    if (m == MPCD_BC_THERMALIZE) {
                        *vx = p->Ubottom + sig * normal01(&nd, &r);
                        *vy = fabs(sig * normal01(&nd, &r));
                    } else if (m == MPCD_BC_BOUNCEBACK) {
                        *vx = 2.0 * p->Ubottom - *vx;
                        *vy = fabs(*vy);
                    } else {
                        *vy = fabs(*vy);
                    }
                    const double dvx = *vx - ox, dvy = *vy - oy;
                    w.nBot += 1;
                    w.dEwall += 0.5 * ((*vx * *vx + *vy * *vy) - (ox * ox + oy * oy));
                    w.dPxBot += dvx;
                    w.dPyBot += fabs(dvy);
                } else {
                    return fail(MPCD_ERR_UNSUPPORTED_BC, "Unsupported boundary_bottom mode");
                }
            }
            if (*yi > Ly) {
                const double ox = *vx, oy = *vy;
                const int m = p->boundary_top;
                if (m == MPCD_BC_PERIODIC) {
                    *yi -= Ly;
                } else if (m == MPCD_BC_THERMALIZE || m == MPCD_BC_BOUNCEBACK || m == MPCD_BC_SPECULAR) {
                    *yi = 2.0 * Ly - *yi;
                    if (m == MPCD_BC_THERMALIZE) {
                        *vx = p->Utop + sig * normal01(&nd, &r);
                        *vy = -fabs(sig * normal01(&nd, &r));
                    } else if (m == MPCD_BC_BOUNCEBACK) {
                        *vx = 2.0 * p->Utop - *vx;
                        *vy = -fabs(*vy);
                    } else {
                        *vy = -fabs(*vy);
                    }
                    const double dvx = *vx - ox, dvy = *vy - oy;
                    w.nTop += 1;
                    w.dEwall += 0.5 * ((*vx * *vx + *vy * *vy) - (ox * ox + oy * oy));
                    w.dPxTop += dvx;
                    w.dPyTop += fabs(dvy);
                } else {
                    return fail(MPCD_ERR_UNSUPPORTED_BC, "Unsupported boundary_top mode");
                }
            }
        }
    }
    (void)bc_side_name;
    for (int i = 0; i < p->n; ++i) {
        double* xi = &x[2 * i];
        if (periodic_x(p)) {
            *xi = *xi - floor(*xi / Lx) * Lx;
        } else {
            if (*xi < 0.0) *xi = 0.0;
            if (*xi > Lx) *xi = Lx;
        }
    }
    for (int i = 0; i < p->n; ++i) {
        double* yi = &x[2 * i + 1];
        if (periodic_y(p)) {
            *yi = *yi - floor(*yi / Ly) * Ly;
        } else {
            if (*yi < 0.0) *yi = 0.0;
            if (*yi > Ly) *yi = Ly;
        }
    }
    if (info) *info = w;
    return MPCD_OK;
}

/* =========================================================================== SRD */

/* src/srd_collision.cpp:9-45 */
void oracle_srd_shift_cells(const P* p, const double* x, uint64_t seed, int32_t* cid) {
    mt64 r;
    mt_seed(&r, seed);
    const double sx = unif(&r, -0.5 * p->a0, 0.5 * p->a0);
    const double sy = unif(&r, -0.5 * p->a0, 0.5 * p->a0);
    for (int i = 0; i < p->n; ++i) {
        double xs = x[2 * i] + sx, ys = x[2 * i + 1] + sy;
        if (periodic_x(p)) {
            xs = xs - floor(xs / p->Lx) * p->Lx;
        } else {
            if (xs < 0.0) xs = 0.0;
            if (xs >= p->Lx) xs = nextafter(p->Lx, 0.0);
        }
        if (periodic_y(p)) {
            ys = ys - floor(ys / p->Ly) * p->Ly;
        } else {
            if (ys < 0.0) ys = 0.0;
            if (ys >= p->Ly) ys = nextafter(p->Ly, 0.0);
        }
        int ix = (int)floor(xs / p->a0), iy = (int)floor(ys / p->a0);
        if (ix < 0) ix = 0;
        if (ix >= p->Nx) ix = p->Nx - 1;
        if (iy < 0) iy = 0;
        if (iy >= p->Ny) iy = p->Ny - 1;
        cid[i] = iy + p->Ny * ix;
    }
}

/* src/srd_collision.cpp:47-140 */
int oracle_srd_collide(const P* p, double* v, const int32_t* cid, uint64_t seed) {
    const int n = p->n, Nc = p->Nc;
    mt64 r;
    mt_seed(&r, seed);
    int* cnt = (int*)calloc((size_t)Nc, sizeof(int));
    double* sum = (double*)calloc(2 * (size_t)Nc, sizeof(double));
    double* u = (double*)calloc(2 * (size_t)Nc, sizeof(double));
    double* th = (double*)calloc((size_t)Nc, sizeof(double));
    double* rel = (double*)calloc(3 * (size_t)n, sizeof(double));
    double* sr2 = (double*)calloc((size_t)Nc, sizeof(double));
    for (int i = 0; i < n; ++i) {
        const int c = cid[i];
        if (c < 0 || c >= Nc) { free(cnt); free(sum); free(u); free(th); free(rel); free(sr2); return fail(MPCD_ERR_INVALID_ARG, "cell id out of range"); }
        cnt[c] += 1;
        sum[2 * c] += v[2 * i];
        sum[2 * c + 1] += v[2 * i + 1];
    }
    for (int c = 0; c < Nc; ++c)
        if (cnt[c] > 0) {
            u[2 * c] = sum[2 * c] / (double)cnt[c];
            u[2 * c + 1] = sum[2 * c + 1] / (double)cnt[c];
        }
    for (int c = 0; c < Nc; ++c)
        if (cnt[c] >= 2) th[c] = p->alpha * ((unif(&r, 0.0, 1.0) < 0.5) ? -1.0 : 1.0);
    for (int i = 0; i < n; ++i) {
        const int c = cid[i];
        const double vxr = v[2 * i] - u[2 * c], vyr = v[2 * i + 1] - u[2 * c + 1];
        const double ct = cos(th[c]), st = sin(th[c]);
        rel[3 * i] = ct * vxr - st * vyr;
        rel[3 * i + 1] = st * vxr + ct * vyr;
        rel[3 * i + 2] = rel[3 * i] * rel[3 * i] + rel[3 * i + 1] * rel[3 * i + 1];
    }
    if (p->useThermostat) {
        for (int i = 0; i < n; ++i) sr2[cid[i]] += rel[3 * i + 2];
        for (int c = 0; c < Nc; ++c) {
            const int dof = 2 * imax(cnt[c] - 1, 0);
            double lam = 1.0;
            if (cnt[c] > 1 && sr2[c] > 0.0) lam = sqrt(((double)dof * p->kBT) / sr2[c]);
            sr2[c] = lam;
        }
        for (int i = 0; i < n; ++i) {
            rel[3 * i] *= sr2[cid[i]];
            rel[3 * i + 1] *= sr2[cid[i]];
        }
    }
    for (int i = 0; i < n; ++i) {
        const int c = cid[i];
        v[2 * i] = u[2 * c] + rel[3 * i];
        v[2 * i + 1] = u[2 * c + 1] + rel[3 * i + 1];
    }
    if (p->keepMeanFlow) {
        double mx = 0.0, my = 0.0;
        for (int i = 0; i < n; ++i) { mx += v[2 * i]; my += v[2 * i + 1]; }
        mx /= (double)n;
        my /= (double)n;
        for (int i = 0; i < n; ++i) { v[2 * i] -= mx; v[2 * i + 1] -= my; }
    }
    free(cnt); free(sum); free(u); free(th); free(rel); free(sr2);
    return MPCD_OK;
}

/* ================================================================== cell fields */

/* src/common_grid.cpp:32-100 */
void oracle_cell_fields(const P* p, const double* x, const double* v, double rhoT, mpcd_cellfields_c* G) {
    const int n = p->n, Nc = p->Nc;
    const double dx = p->Lx / (double)p->Nx, dy = p->Ly / (double)p->Ny, Vc = dx * dy;
    int32_t* N = (int32_t*)calloc((size_t)Nc, sizeof(int32_t));
    double* f = (double*)calloc(11 * (size_t)Nc, sizeof(double));
    double *Ux = f, *Uy = f + Nc, *Px = f + 2 * Nc, *Py = f + 3 * Nc, *T = f + 4 * Nc, *rho = f + 5 * Nc,
           *Pk = f + 6 * Nc, *Pv = f + 7 * Nc, *PP = f + 8 * Nc, *rt = f + 9 * Nc, *s2 = f + 10 * Nc;
    int* cid = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) {
        const int c = cid[i] = cell_of(x[2 * i], x[2 * i + 1], p);
        N[c] += 1;
        Px[c] += v[2 * i];
        Py[c] += v[2 * i + 1];
    }
    for (int c = 0; c < Nc; ++c) {
        if (N[c] > 0) {
            Ux[c] = Px[c] / (double)N[c];
            Uy[c] = Py[c] / (double)N[c];
        }
        rho[c] = (double)N[c] / Vc;
        rt[c] = rhoT;
    }
    for (int i = 0; i < n; ++i) {
        const int c = cid[i];
        const double ax = v[2 * i] - Ux[c], ay = v[2 * i + 1] - Uy[c];
        s2[c] += ax * ax + ay * ay;
    }
    for (int c = 0; c < Nc; ++c) {
        const int dof = 2 * imax(N[c] - 1, 0);
        if (dof > 0) {
            T[c] = s2[c] / (double)dof;
            Pk[c] = rho[c] * T[c];
        } else {
            T[c] = 0.0;
            Pk[c] = 0.0;
        }
        Pv[c] = p->Kvirial * (rho[c] - rt[c]);
        PP[c] = Pk[c] + Pv[c];
    }
    if (G->N) memcpy(G->N, N, sizeof(int32_t) * (size_t)Nc);
    double* dst[10] = {G->Ux, G->Uy, G->Px, G->Py, G->T, G->rho, G->Pkin, G->Pvir, G->P, G->rhoTarget};
    for (int k = 0; k < 10; ++k)
        if (dst[k]) memcpy(dst[k], f + (size_t)k * Nc, sizeof(double) * (size_t)Nc);
    free(N); free(f); free(cid);
}

/* ================================================================== zone layout */

typedef struct {
    int xs, xe, ys, ye;
} rect;

/* src/zone_pass.cpp:160-171 */
static int start_indices(int N, int tile, int off, int* out) {
    int m = 0;
    out[m++] = 0;
    for (int s = off; s < N; s += tile)
        if (s > 0 && s < N) out[m++] = s; /* increasing already: sort/unique are no-ops */
    return m;
}

/* src/zone_pass.cpp:173-221; owner may be NULL. Returns the zone count. */
static int build_layout(const P* p, int mode, rect** zones_out, int32_t* owner) {
    if (mode == MPCD_LAYOUT_SINGLE_FULL || p->zoneSingleFullDomainMode) {
        rect* z = (rect*)malloc(sizeof(rect));
        z->xs = 0; z->xe = p->Nx; z->ys = 0; z->ye = p->Ny;
        if (owner) for (int c = 0; c < p->Nc; ++c) owner[c] = 1;
        *zones_out = z;
        return 1;
    }
    const int offx = (mode == MPCD_LAYOUT_SHIFTED) ? p->zoneTileNx / 2 : 0;
    const int offy = (mode == MPCD_LAYOUT_SHIFTED) ? p->zoneTileNy / 2 : 0;
    int* xst = (int*)malloc(sizeof(int) * (size_t)(p->Nx + 2));
    int* yst = (int*)malloc(sizeof(int) * (size_t)(p->Ny + 2));
    const int nxs = start_indices(p->Nx, p->zoneTileNx, offx, xst);
    const int nys = start_indices(p->Ny, p->zoneTileNy, offy, yst);
    rect* z = (rect*)malloc(sizeof(rect) * (size_t)(nxs * nys));
    int id = 0;
    for (int a = 0; a < nys; ++a)
        for (int b = 0; b < nxs; ++b) {
            rect q;
            q.xs = xst[b]; q.xe = imin(xst[b] + p->zoneTileNx, p->Nx);
            q.ys = yst[a]; q.ye = imin(yst[a] + p->zoneTileNy, p->Ny);
            z[id++] = q;
            if (owner)
                for (int ix = q.xs; ix < q.xe; ++ix)
                    for (int iy = q.ys; iy < q.ye; ++iy) owner[iy + p->Ny * ix] = id;
        }
    free(xst); free(yst);
    *zones_out = z;
    return id;
}

int oracle_zone_owner_map(const P* p, int mode, int32_t* owner) {
    rect* z = NULL;
    const int nz = build_layout(p, mode, &z, owner);
    free(z);
    return nz;
}

/* =============================================================== zone kernel */

/* growable int list */
typedef struct {
    int* a;
    int n, cap;
} ilist;

static void il_push(ilist* l, int v) {
    if (l->n == l->cap) {
        l->cap = l->cap ? 2 * l->cap : 16;
        l->a = (int*)realloc(l->a, sizeof(int) * (size_t)l->cap);
    }
    l->a[l->n++] = v;
}

typedef struct {
    const P* p;
    rect R;
    int TX, TY;             /* rectangle size */
    const int32_t* cnt_in;  /* snapshot counts, all cells */
    int* cnt;               /* live counts of zone cells, local index */
    ilist* parts;           /* live particle lists of zone cells (particle ids) */
    char *recv, *bb, *skip; /* correction masks (local) */
    double *lowA, *highA;   /* per-pass threshold maps (local) */
    double *Nsm;            /* smoothed occupancy on the rectangle grown by 1 (non-periodic) */
    double highThr, lowThrBulk;
    mt64 rng;
    double* x;              /* output positions (particle-id order) */
    int movedDense, movedSparse;
} zctx;

static int in_zone(const zctx* z, int ix, int iy) { return ix >= z->R.xs && ix < z->R.xe && iy >= z->R.ys && iy < z->R.ye; }
static int loc(const zctx* z, int ix, int iy) { return (ix - z->R.xs) * z->TY + (iy - z->R.ys); }
static void cell_xy(const P* p, int c, int* ix, int* iy) { *ix = c / p->Ny; *iy = c - (*ix) * p->Ny; }
static int cnt_at(const zctx* z, int ix, int iy) {
    return in_zone(z, ix, iy) ? z->cnt[loc(z, ix, iy)] : z->cnt_in[iy + z->p->Ny * ix];
}
static int cnt_c(const zctx* z, int c) { int ix, iy; cell_xy(z->p, c, &ix, &iy); return cnt_at(z, ix, iy); }

/* src/zone_pass.cpp:246-261 */
static int shift_index(const P* p, int iy, int ix, int dy, int dx, int* jy, int* jx) {
    *jy = iy + dy;
    if (periodic_y(p)) *jy = wrap_index(*jy, p->Ny);
    else if (*jy < 0 || *jy >= p->Ny) return 0;
    *jx = ix + dx;
    if (periodic_x(p)) *jx = wrap_index(*jx, p->Nx);
    else if (*jx < 0 || *jx >= p->Nx) return 0;
    return 1;
}

/* src/zone_pass.cpp:229-244 */
static void minimal_step(const P* p, int src, int dst, int* ddx, int* ddy) {
    int sx, sy, tx, ty;
    cell_xy(p, src, &sx, &sy);
    cell_xy(p, dst, &tx, &ty);
    int a = tx - sx, b = ty - sy;
    if (periodic_x(p)) { if (a > p->Nx / 2) a -= p->Nx; if (a < -p->Nx / 2) a += p->Nx; }
    if (periodic_y(p)) { if (b > p->Ny / 2) b -= p->Ny; if (b < -p->Ny / 2) b += p->Ny; }
    *ddx = a; *ddy = b;
}

/* Nsm at (ix, iy): src/zone_pass.cpp:296-319 (3x3 [1 2 1]^2/16, non-periodic, renormalised) */
static double smooth_at(const zctx* z, int ix, int iy) {
    static const double K[9] = {1.0 / 16.0, 2.0 / 16.0, 1.0 / 16.0, 2.0 / 16.0, 4.0 / 16.0, 2.0 / 16.0, 1.0 / 16.0, 2.0 / 16.0, 1.0 / 16.0};
    const P* p = z->p;
    double acc = 0.0, ws = 0.0;
    int kk = 0;
    for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx, ++kk) {
            const int jy = iy + dy, jx = ix + dx;
            if (jy < 0 || jy >= p->Ny || jx < 0 || jx >= p->Nx) continue;
            acc += K[kk] * (double)cnt_at(z, jx, jy);
            ws += K[kk];
        }
    return acc / dmax(ws, 1e-30);
}

/* Nsm over the rectangle grown by one cell (wrapped coordinates where periodic) */
static int nsm_idx(const zctx* z, int ix, int iy) {
    /* (ix, iy) is a cell within Chebyshev distance 1 of the rectangle, possibly wrapped */
    const P* p = z->p;
    int lx = ix - (z->R.xs - 1), ly = iy - (z->R.ys - 1);
    if (lx < 0) lx += p->Nx;
    if (lx >= z->TX + 2) lx -= p->Nx;
    if (ly < 0) ly += p->Ny;
    if (ly >= z->TY + 2) ly -= p->Ny;
    return lx * (z->TY + 2) + ly;
}
static void compute_nsm(zctx* z) {
    const P* p = z->p;
    for (int lx = 0; lx < z->TX + 2; ++lx)
        for (int ly = 0; ly < z->TY + 2; ++ly) {
            int ix = z->R.xs - 1 + lx, iy = z->R.ys - 1 + ly;
            double val = 0.0;
            if (periodic_x(p)) ix = wrap_index(ix, p->Nx);
            if (periodic_y(p)) iy = wrap_index(iy, p->Ny);
            if (ix >= 0 && ix < p->Nx && iy >= 0 && iy < p->Ny) val = smooth_at(z, ix, iy);
            z->Nsm[lx * (z->TY + 2) + ly] = val;
        }
}
static double nsm(const zctx* z, int c) { int ix, iy; cell_xy(z->p, c, &ix, &iy); return z->Nsm[nsm_idx(z, ix, iy)]; }

/* threshold maps for zone cells: src/zone_pass.cpp:321-345 and :715-725 */
static void build_maps(zctx* z) {
    const P* p = z->p;
    const double lowFrac = 1.0 / (1.0 + p->coef), highFrac = 1.0 + p->coef;
    if (p->useLocalFluidFractionThresholds) compute_nsm(z);
    for (int ix = z->R.xs; ix < z->R.xe; ++ix)
        for (int iy = z->R.ys; iy < z->R.ye; ++iy) {
            const int l = loc(z, ix, iy);
            double f = 1.0;
            if (p->useLocalFluidFractionThresholds) {
                const double fraw = z->Nsm[nsm_idx(z, ix, iy)] / dmax(p->gamma, 1e-12);
                const double g = p->fluidFracGain * fraw;
                f = (g < 0.0) ? 0.0 : ((1.0 < g) ? 1.0 : g);
            }
            const double gl = p->gamma * f;
            double lo = dmax(lowFrac * gl, p->lowThrFloor), hi = dmax(highFrac * gl, p->highThrFloor);
            if (z->cnt[l] > 0) { lo = z->lowThrBulk; hi = z->highThr; }
            z->lowA[l] = lo;
            z->highA[l] = hi;
        }
}

static double mapval(const zctx* z, const double* map, int c) { int ix, iy; cell_xy(z->p, c, &ix, &iy); return map[loc(z, ix, iy)]; }

/* admissible_dense_targets_rangeR (src/zone_pass.cpp:413-434) followed by the zone filter of
 * src/zone_pass.cpp:611; the unfiltered entries never influence anything. */
static int admissible(const zctx* z, int c, const double* map, int* out) {
    const P* p = z->p;
    int ix, iy, m = 0;
    cell_xy(p, c, &ix, &iy);
    for (int dy = -2; dy <= 2; ++dy)
        for (int dx = -2; dx <= 2; ++dx) {
            if (dx == 0 && dy == 0) continue;
            int jy, jx;
            if (!shift_index(p, iy, ix, dy, dx, &jy, &jx)) continue;
            if (!in_zone(z, jx, jy)) continue;
            const int nb = jy + p->Ny * jx;
            if ((double)cnt_at(z, jx, jy) < map[loc(z, jx, jy)]) {
                int dup = 0;
                for (int q = 0; q < m; ++q) dup |= (out[q] == nb);
                if (!dup) out[m++] = nb;
            }
        }
    return m;
}

typedef struct {
    int nb;
    double deficitNeg, inwardNeg;
    int cnt, cheb, dist2;
    double tie;
} cand;

static int cand_less(const cand* a, const cand* b) {
    if (a->deficitNeg != b->deficitNeg) return a->deficitNeg < b->deficitNeg;
    if (a->inwardNeg != b->inwardNeg) return a->inwardNeg < b->inwardNeg;
    if (a->cnt != b->cnt) return a->cnt < b->cnt;
    if (a->cheb != b->cheb) return a->cheb < b->cheb;
    if (a->dist2 != b->dist2) return a->dist2 < b->dist2;
    return a->tie < b->tie;
}

/* rank_dense_targets_unified (src/zone_pass.cpp:436-490); inwardWeight is 0 at the only
 * call site (src/zone_pass.cpp:740-741). std::sort on <= 16 elements is libstdc++'s
 * insertion sort, i.e. stable. */
static int rank_dense(zctx* z, int c, const int* adm, int m, const double* map, int* ordered) {
    if (m == 0) return 0;
    const P* p = z->p;
    cand bins[8][24];
    int nb_[8] = {0};
    const int startBin = (int)unif_int(&z->rng, 1, 8) - 1;
    for (int k = 0; k < m; ++k) {
        const int nb = adm[k];
        int dx, dy;
        minimal_step(p, c, nb, &dx, &dy);
        const double ang = atan2((double)dy, (double)dx);
        int ib = (int)floor((ang + M_PI) / (2.0 * M_PI / 8.0));
        ib = ((ib % 8) + 8) % 8;
        const double deficit = dmax(0.0, mapval(z, map, nb) - (double)cnt_c(z, nb));
        cand cd;
        cd.nb = nb;
        cd.deficitNeg = -deficit;
        cd.inwardNeg = -0.0 * 0.0;
        cd.cnt = cnt_c(z, nb);
        cd.cheb = imax(abs(dx), abs(dy));
        cd.dist2 = dx * dx + dy * dy;
        cd.tie = unif(&z->rng, 0.0, 1.0);
        bins[ib][nb_[ib]++] = cd;
    }
    for (int b = 0; b < 8; ++b) /* stable insertion sort */
        for (int i = 1; i < nb_[b]; ++i) {
            cand v = bins[b][i];
            int j = i;
            while (j > 0 && cand_less(&v, &bins[b][j - 1])) { bins[b][j] = bins[b][j - 1]; --j; }
            bins[b][j] = v;
        }
    int taken[8] = {0}, out = 0, keep = 1;
    while (keep) {
        keep = 0;
        for (int s = 0; s < 8; ++s) {
            const int ib = (startBin + s) % 8;
            if (taken[ib] >= nb_[ib]) continue;
            ordered[out++] = bins[ib][taken[ib]++].nb;
            keep = 1;
        }
    }
    return out;
}

/* sample_in_cell (src/zone_pass.cpp:280-294) applied to particle pid */
static void place_in_cell(zctx* z, int cell, int pid) {
    const P* p = z->p;
    int ix, iy;
    cell_xy(p, cell, &ix, &iy);
    const double dx = p->Lx / (double)p->Nx, dy = p->Ly / (double)p->Ny;
    const double x0 = (double)ix * dx, y0 = (double)iy * dy;
    const double ux = unif(&z->rng, 0.0, 1.0);
    const double uy = unif(&z->rng, 0.0, 1.0);
    z->x[2 * pid] = x0 + dx * ux;
    z->x[2 * pid + 1] = y0 + dy * uy;
}

static void push_unique(int* a, int* m, int v) {
    for (int q = 0; q < *m; ++q) if (a[q] == v) return;
    a[(*m)++] = v;
}

/* spread_particles_from_dense_source_round_robin (src/zone_pass.cpp:527-589). The sampled
 * positions of one batch are drawn in particle order, x then y (sample_in_cell). Returns the
 * number of unique receiving targets written to recv. */
static int spread(zctx* z, int src, const int* T, int nT, const double* map, int needOut, int* recv, int* moved) {
    *moved = 0;
    if (needOut <= 0 || nT == 0) return 0;
    ilist* S = &z->parts[loc(z, src / z->p->Ny, src % z->p->Ny)];
    if (S->n == 0) return 0;
    int head = 0; /* idsAvail = S->a[head .. S->n) */
    int nrecv = 0;
    while (needOut > 0 && head < S->n) {
        int progressed = 0;
        for (int kk = 0; kk < nT; ++kk) {
            const int nb = T[kk];
            const int deficit = imax(0, (int)floor(mapval(z, map, nb) - (double)cnt_c(z, nb)));
            if (deficit <= 0) continue;
            int remaining = 0;
            for (int jj = kk; jj < nT; ++jj) {
                const int dj = imax(0, (int)floor(mapval(z, map, T[jj]) - (double)cnt_c(z, T[jj])));
                if (dj > 0) ++remaining;
            }
            const int quota = imax(1, (int)ceil((double)needOut / imax(1, remaining)));
            const int nt = imax(1, imin(imin(quota, deficit), imin(needOut, S->n - head)));
            int bx, by;
            cell_xy(z->p, nb, &bx, &by);
            ilist* D = &z->parts[loc(z, bx, by)];
            for (int q = 0; q < nt; ++q) {
                const int pid = S->a[head + q];
                place_in_cell(z, nb, pid);
                il_push(D, pid);
            }
            head += nt;
            z->cnt[loc(z, bx, by)] += nt;
            push_unique(recv, &nrecv, nb); /* unique_stable of the batch targets */
            *moved += nt;
            needOut -= nt;
            progressed = 1;
            if (needOut <= 0 || head >= S->n) break;
        }
        if (!progressed) break;
    }
    if (*moved > 0) {
        memmove(S->a, S->a + head, sizeof(int) * (size_t)(S->n - head));
        S->n -= head;
        z->cnt[loc(z, src / z->p->Ny, src % z->p->Ny)] = S->n;
        return nrecv;
    }
    return 0;
}

/* update_transfer_correction_masks (src/zone_pass.cpp:492-525), forceSkip = false */
static void update_masks(zctx* z, int src, const int* recv, int nrecv, const char* bulkBefore) {
    int t[64], nt = 0;
    push_unique(t, &nt, src);
    for (int q = 0; q < nrecv; ++q) push_unique(t, &nt, recv[q]);
    int all = 1;
    for (int q = 0; q < nt; ++q) {
        int ix, iy;
        cell_xy(z->p, t[q], &ix, &iy);
        if (!bulkBefore[loc(z, ix, iy)]) { all = 0; break; }
    }
    for (int q = 0; q < nt; ++q) {
        int ix, iy;
        cell_xy(z->p, t[q], &ix, &iy);
        const int l = loc(z, ix, iy);
        if (all) z->bb[l] = 1;
        else { z->skip[l] = 1; z->bb[l] = 0; }
    }
}

/* inward_direction_from_local_gradient (src/zone_pass.cpp:375-411) */
static void inward_dir(const zctx* z, int c, double* gx, double* gy) {
    const P* p = z->p;
    int ix, iy;
    cell_xy(p, c, &ix, &iy);
#define NS(jx, jy) z->Nsm[nsm_idx(z, (jx), (jy))]
    if (periodic_x(p)) *gx = 0.5 * (NS(wrap_index(ix + 1, p->Nx), iy) - NS(wrap_index(ix - 1, p->Nx), iy));
    else if (ix == 0) *gx = NS(ix + 1, iy) - NS(ix, iy);
    else if (ix == p->Nx - 1) *gx = NS(ix, iy) - NS(ix - 1, iy);
    else *gx = 0.5 * (NS(ix + 1, iy) - NS(ix - 1, iy));
    if (periodic_y(p)) *gy = 0.5 * (NS(ix, wrap_index(iy + 1, p->Ny)) - NS(ix, wrap_index(iy - 1, p->Ny)));
    else if (iy == 0) *gy = NS(ix, iy + 1) - NS(ix, iy);
    else if (iy == p->Ny - 1) *gy = NS(ix, iy) - NS(ix, iy - 1);
    else *gy = 0.5 * (NS(ix, iy + 1) - NS(ix, iy - 1));
#undef NS
}

/* rank_admissible_neighbors_inward (src/zone_pass.cpp:636-667); the sort is on <= 8
 * elements (libstdc++ insertion sort, stable) */
static int rank_inward(zctx* z, int c, int* don, int m, double gx, double gy) {
    if (m == 0) return 0;
    const P* p = z->p;
    shuffle_ints(don, m, &z->rng);
    const double ndir = hypot(gx, gy);
    normal_st nd = {0.0, 0};
    double score[8];
    int ord[8];
    for (int k = 0; k < m; ++k) {
        int dx, dy;
        minimal_step(p, c, don[k], &dx, &dy);
        const double nstep = hypot((double)dx, (double)dy);
        double align = 0.0;
        if (ndir >= 1e-14 && nstep >= 1e-14) align = ((double)dx * gx + (double)dy * gy) / (ndir * nstep);
        const double noise = 1e-9 * normal01(&nd, &z->rng);
        score[k] = 100.0 * align + nsm(z, don[k]) + noise;
        ord[k] = don[k];
    }
    for (int i = 1; i < m; ++i) {
        const double sv = score[i];
        const int ov = ord[i];
        int j = i;
        while (j > 0 && sv > score[j - 1]) { score[j] = score[j - 1]; ord[j] = ord[j - 1]; --j; }
        score[j] = sv;
        ord[j] = ov;
    }
    memcpy(don, ord, sizeof(int) * (size_t)m);
    return m;
}

/* occupancy_thresholds (src/zone_pass.cpp:347-366) */
static void thresholds(const P* p, double* highThr, double* lowThrBulk) {
    const double g = p->gamma, cf = p->coef;
    *highThr = (p->highMode == MPCD_THR_ONE_PLUS_COEF) ? g * (1.0 + cf) : g + g * cf;
    *lowThrBulk = (p->lowMode == MPCD_THR_ONE_PLUS_COEF) ? g / (1.0 + cf) : g - g * cf;
    if (isfinite(p->lowThrBulkOverride)) *lowThrBulk = p->lowThrBulkOverride;
}

/* run_zone_kernel (src/zone_pass.cpp:669-973) on the snapshot, zone-locally. Writes the new
 * positions into x and applies the momentum correction to v for the zone's particles.
 * stats4/stats5 = the kernel's stats[4], stats[5]. */
static void zone_kernel(const P* p, rect R, const int32_t* cnt_in, const int32_t* start_in, const int32_t* ids_in,
                        const double* vin, double* x, double* v, uint64_t seed, int* mD, int* mS, double* st4, double* st5) {
    zctx Z;
    memset(&Z, 0, sizeof Z);
    zctx* z = &Z;
    z->p = p;
    z->R = R;
    z->TX = R.xe - R.xs;
    z->TY = R.ye - R.ys;
    const int nl = z->TX * z->TY;
    z->cnt_in = cnt_in;
    z->cnt = (int*)calloc((size_t)nl, sizeof(int));
    z->parts = (ilist*)calloc((size_t)nl, sizeof(ilist));
    z->recv = (char*)calloc((size_t)nl, 1);
    z->bb = (char*)calloc((size_t)nl, 1);
    z->skip = (char*)calloc((size_t)nl, 1);
    z->lowA = (double*)calloc((size_t)nl, sizeof(double));
    z->highA = (double*)calloc((size_t)nl, sizeof(double));
    z->Nsm = (double*)calloc((size_t)(z->TX + 2) * (size_t)(z->TY + 2), sizeof(double));
    char* bulkBefore = (char*)calloc((size_t)nl, 1);
    char* changed = (char*)calloc((size_t)nl, 1);
    z->x = x;
    thresholds(p, &z->highThr, &z->lowThrBulk);
    mt_seed(&z->rng, seed);
    for (int ix = R.xs; ix < R.xe; ++ix)
        for (int iy = R.ys; iy < R.ye; ++iy) {
            const int c = iy + p->Ny * ix, l = loc(z, ix, iy);
            z->cnt[l] = cnt_in[c];
            for (int k = start_in[c]; k < start_in[c + 1]; ++k) il_push(&z->parts[l], ids_in[k]);
        }
    int* dense = (int*)malloc(sizeof(int) * (size_t)nl);
    int adm[24], ord[24], recv[64], recv2[64], T2[24];
    for (int pass = 0; pass < p->maxRedistribPasses; ++pass) {
        build_maps(z);
        for (int l = 0; l < nl; ++l) bulkBefore[l] = z->cnt[l] > 0;
        int nd = 0;
        for (int ix = R.xs; ix < R.xe; ++ix)
            for (int iy = R.ys; iy < R.ye; ++iy) {
                const int l = loc(z, ix, iy);
                if ((double)z->cnt[l] > z->highA[l]) dense[nd++] = iy + p->Ny * ix;
            }
        shuffle_ints(dense, nd, &z->rng);
        for (int q = 0; q < nd; ++q) {
            const int c = dense[q];
            int ix, iy;
            cell_xy(p, c, &ix, &iy);
            const int l = loc(z, ix, iy);
            const int ncc = z->cnt[l];
            if (ncc <= 0) continue;
            const double hl = z->highA[l];
            if ((double)ncc <= hl) continue;
            /* redistribute_dense_cell_at_range_zone_local (src/zone_pass.cpp:591-634) */
            int nrecv = 0, moved = 0, movedNow = 0;
            const int needOut = imax(0, (int)ceil((double)z->cnt[l] - hl));
            if (needOut > 0) {
                int m = admissible(z, c, z->lowA, adm);
                int nT = rank_dense(z, c, adm, m, z->lowA, ord);
                int nr = spread(z, c, ord, nT, z->lowA, needOut, recv2, &movedNow);
                for (int k = 0; k < nr; ++k) push_unique(recv, &nrecv, recv2[k]);
                moved += movedNow;
                const int remainingOut = imax(0, (int)ceil((double)z->cnt[l] - hl));
                if (remainingOut > 0) {
                    m = admissible(z, c, z->highA, adm);
                    nT = rank_dense(z, c, adm, m, z->highA, T2);
                    nr = spread(z, c, T2, nT, z->highA, remainingOut, recv2, &movedNow);
                    for (int k = 0; k < nr; ++k) push_unique(recv, &nrecv, recv2[k]);
                    moved += movedNow;
                }
            }
            for (int k = 0; k < nrecv; ++k) {
                int rx, ry;
                cell_xy(p, recv[k], &rx, &ry);
                z->recv[loc(z, rx, ry)] = 1;
                changed[loc(z, rx, ry)] = 1;
            }
            if (moved > 0) changed[l] = 1;
            update_masks(z, c, recv, nrecv, bulkBefore);
            z->movedDense += moved;
        }
    }
    /* sparse phase: src/zone_pass.cpp:783-854 */
    compute_nsm(z);
    build_maps(z);
    for (int l = 0; l < nl; ++l) bulkBefore[l] = z->cnt[l] > 0;
    int nlow = 0;
    for (int ix = R.xs; ix < R.xe; ++ix)
        for (int iy = R.ys; iy < R.ye; ++iy) {
            const int l = loc(z, ix, iy);
            if (z->cnt[l] > 0 && (double)z->cnt[l] < z->lowA[l]) dense[nlow++] = iy + p->Ny * ix;
        }
    shuffle_ints(dense, nlow, &z->rng);
    const int lowInt = (int)ceil(z->lowThrBulk);
    for (int q = 0; q < nlow; ++q) {
        const int c = dense[q];
        int ix, iy;
        cell_xy(p, c, &ix, &iy);
        const int l = loc(z, ix, iy);
        const int ncc = z->cnt[l];
        if (ncc <= 0) continue;
        if (z->parts[l].n == 0) continue;
        /* local_neighbors_in_zone (src/zone_pass.cpp:263-278), range 1 */
        int neigh[8], nn = 0;
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                if (dx == 0 && dy == 0) continue;
                int jy, jx;
                if (!shift_index(p, iy, ix, dy, dx, &jy, &jx)) continue;
                if (in_zone(z, jx, jy)) push_unique(neigh, &nn, jy + p->Ny * jx);
            }
        if (nn == 0) continue;
        int need = imax(0, lowInt - ncc);
        if (need <= 0) continue;
        int don[8], ndn = 0;
        for (int k = 0; k < nn; ++k)
            if (cnt_c(z, neigh[k]) > lowInt) don[ndn++] = neigh[k];
        if (ndn == 0) continue;
        double gx, gy;
        inward_dir(z, c, &gx, &gy);
        rank_inward(z, c, don, ndn, gx, gy);
        for (int k = 0; k < ndn; ++k) {
            const int d = don[k];
            int dx_, dy_;
            cell_xy(p, d, &dx_, &dy_);
            const int ld = loc(z, dx_, dy_);
            ilist* Dl = &z->parts[ld];
            if (Dl->n == 0) continue;
            const int avail = z->cnt[ld] - lowInt;
            if (avail <= 0) continue;
            const int nt = imin(imin(need, avail), Dl->n);
            if (nt <= 0) continue;
            shuffle_ints(Dl->a, Dl->n, &z->rng);
            for (int t = 0; t < nt; ++t) {
                const int pid = Dl->a[t];
                place_in_cell(z, c, pid);
                il_push(&z->parts[l], pid);
            }
            memmove(Dl->a, Dl->a + nt, sizeof(int) * (size_t)(Dl->n - nt));
            Dl->n -= nt;
            z->cnt[ld] = Dl->n;
            z->cnt[l] += nt;
            z->recv[l] = 1;
            changed[l] = 1;
            changed[ld] = 1;
            int one[1] = {c};
            update_masks(z, d, one, 1, bulkBefore);
            z->movedSparse += nt;
            need -= nt;
            if (need <= 0) break;
        }
    }
    /* momentum correction: src/zone_pass.cpp:870-922 (cells in ascending index order) */
    double accDU = 0.0, dUmax = 0.0;
    int nDU = 0;
    for (int ix = R.xs; ix < R.xe; ++ix)
        for (int iy = R.ys; iy < R.ye; ++iy) {
            const int c = iy + p->Ny * ix, l = loc(z, ix, iy);
            const ilist* L = &z->parts[l];
            if (L->n == 0) continue;
            double pbx = 0.0, pby = 0.0, pax = 0.0, pay = 0.0;
            for (int k = start_in[c]; k < start_in[c + 1]; ++k) { pbx += vin[2 * ids_in[k]]; pby += vin[2 * ids_in[k] + 1]; }
            for (int k = 0; k < L->n; ++k) { pax += vin[2 * L->a[k]]; pay += vin[2 * L->a[k] + 1]; }
            const double dPx = pbx - pax, dPy = pby - pay;
            const double dux = dPx / (double)L->n, duy = dPy / (double)L->n;
            const double du2 = dux * dux + duy * duy;
            dUmax = dmax(dUmax, sqrt(du2));
            if (du2 > 0.0) { accDU += du2; ++nDU; }
            int doCorr = p->enableMomentumCorrectionPostRedistribution;
            if (doCorr && z->skip[l]) doCorr = 0;
            if (doCorr && z->recv[l] && !z->bb[l]) doCorr = 0;
            for (int k = 0; k < L->n; ++k) {
                const int id = L->a[k];
                if (doCorr && (dux != 0.0 || duy != 0.0)) {
                    v[2 * id] = vin[2 * id] + dux;
                    v[2 * id + 1] = vin[2 * id + 1] + duy;
                } else {
                    v[2 * id] = vin[2 * id];
                    v[2 * id + 1] = vin[2 * id + 1];
                }
            }
        }
    *st4 = (nDU > 0) ? sqrt(accDU / (double)nDU) : 0.0;
    *st5 = (nDU > 0) ? dUmax : 0.0;
    *mD = z->movedDense;
    *mS = z->movedSparse;
    for (int l = 0; l < nl; ++l) free(z->parts[l].a);
    free(z->cnt); free(z->parts); free(z->recv); free(z->bb); free(z->skip);
    free(z->lowA); free(z->highA); free(z->Nsm); free(bulkBefore); free(changed); free(dense);
}

static int check_pass_params(const P* p) {
    if (!p->useIncompressibleRedistribution || !p->useZoneRedistribution)
        return fail(MPCD_ERR_INVALID_ARG, "run_zone_pass_snapshot_impl requires useIncompressibleRedistribution=true and useZoneRedistribution=true");
    if (p->redistributionEnableSurfaceTopology || p->redistributionWallWettingEnabled || p->useInterfaceVelocityReorientation)
        return fail(MPCD_ERR_INVALID_ARG, "run_zone_pass_snapshot_impl is restricted to no surface / no wetting / no reorientation");
    if (p->zoneTileNx < 1 || p->zoneTileNy < 1) return fail(MPCD_ERR_INVALID_ARG, "zone tiles must be >= 1");
    return MPCD_OK;
}

/* run_zone_pass_snapshot_impl (src/zone_pass_openmp.cpp:34-172): every zone works on the
 * pass input; the last zone (in id order) whose rectangle holds a particle's input cell
 * provides its output (the serial merge of :146-153). */
int oracle_zone_pass(const P* p, const double* xin, const double* vin, double* xout, double* vout, int mode,
                     uint64_t seedBase, mpcd_pass_metrics_c* m) {
    const int rc = check_pass_params(p);
    if (rc) return rc;
    const int n = p->n, Nc = p->Nc;
    int32_t* cid = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    int32_t* cnt = (int32_t*)calloc((size_t)Nc, sizeof(int32_t));
    int32_t* start = (int32_t*)calloc((size_t)Nc + 1, sizeof(int32_t));
    int32_t* ids = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    int32_t* owner = (int32_t*)malloc(sizeof(int32_t) * (size_t)Nc);
    oracle_cell_ids(p, xin, cid);
    for (int i = 0; i < n; ++i) cnt[cid[i]]++;
    for (int c = 0; c < Nc; ++c) start[c + 1] = start[c] + cnt[c];
    int32_t* cur = (int32_t*)malloc(sizeof(int32_t) * (size_t)Nc);
    memcpy(cur, start, sizeof(int32_t) * (size_t)Nc);
    for (int i = 0; i < n; ++i) ids[cur[cid[i]]++] = i; /* ascending particle id per cell */
    rect* zones = NULL;
    const int nz = build_layout(p, mode, &zones, owner);
    double* xw = (double*)malloc(sizeof(double) * 2 * (size_t)(n > 0 ? n : 1));
    double* vw = (double*)malloc(sizeof(double) * 2 * (size_t)(n > 0 ? n : 1));
    memcpy(xout, xin, sizeof(double) * 2 * (size_t)n);
    memcpy(vout, vin, sizeof(double) * 2 * (size_t)n);
    int totD = 0, totS = 0, corrCount = 0;
    double corrAcc = 0.0, corrMax = 0.0;
    for (int iz = 0; iz < nz; ++iz) {
        const rect R = zones[iz];
        /* the kernel writes only particles of its rectangle; start from the input there */
        for (int ix = R.xs; ix < R.xe; ++ix)
            for (int iy = R.ys; iy < R.ye; ++iy) {
                const int c = iy + p->Ny * ix;
                for (int k = start[c]; k < start[c + 1]; ++k) {
                    const int id = ids[k];
                    xw[2 * id] = xin[2 * id]; xw[2 * id + 1] = xin[2 * id + 1];
                }
            }
        int mD = 0, mS = 0;
        double s4 = 0.0, s5 = 0.0;
        zone_kernel(p, R, cnt, start, ids, vin, xw, vw, seedBase + 104729ULL * (uint64_t)(iz + 1), &mD, &mS, &s4, &s5);
        for (int ix = R.xs; ix < R.xe; ++ix)
            for (int iy = R.ys; iy < R.ye; ++iy) {
                const int c = iy + p->Ny * ix;
                if (owner[c] != iz + 1) continue;
                for (int k = start[c]; k < start[c + 1]; ++k) {
                    const int id = ids[k];
                    xout[2 * id] = xw[2 * id]; xout[2 * id + 1] = xw[2 * id + 1];
                    vout[2 * id] = vw[2 * id]; vout[2 * id + 1] = vw[2 * id + 1];
                }
            }
        totD += mD;
        totS += mS;
        if (s4 > 0.0) { corrAcc += s4 * s4; ++corrCount; }
        corrMax = dmax(corrMax, s5);
    }
    if (m) {
        memset(m, 0, sizeof *m);
        m->nZones = nz;
        m->nThreadsRequested = 1;
        m->nThreadsUsed = 1;
        m->nParticlesMovedDense = totD;
        m->nParticlesMovedSparse = totS;
        m->corrRmsDU = (corrCount > 0) ? sqrt(corrAcc / (double)corrCount) : 0.0;
        m->corrMaxDU = corrMax;
    }
    free(cid); free(cnt); free(start); free(ids); free(owner); free(cur); free(zones); free(xw); free(vw);
    return MPCD_OK;
}

/* run_zone_pass (src/zone_pass.cpp:1096-1163): the zones run one after another, each on the
 * state the previous ones left (cell lists rebuilt from the current positions, ascending
 * particle id), moving and correcting the particles of its rectangle in place. */
int oracle_zone_pass_serial(const P* p, const double* xin, const double* vin, double* xout, double* vout, int mode,
                            uint64_t seedBase, mpcd_pass_metrics_c* m) {
    int rc = check_pass_params(p);
    if (rc) return rc;
    const int n = p->n, Nc = p->Nc;
    int32_t* cid = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    int32_t* cnt = (int32_t*)calloc((size_t)Nc, sizeof(int32_t));
    int32_t* start = (int32_t*)calloc((size_t)Nc + 1, sizeof(int32_t));
    int32_t* cur = (int32_t*)malloc(sizeof(int32_t) * (size_t)Nc);
    int32_t* ids = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    int32_t* owner = (int32_t*)malloc(sizeof(int32_t) * (size_t)Nc);
    double* vsnap = (double*)malloc(sizeof(double) * 2 * (size_t)(n > 0 ? n : 1));
    rect* zones = NULL;
    const int nz = build_layout(p, mode, &zones, owner);
    memcpy(xout, xin, sizeof(double) * 2 * (size_t)n);
    memcpy(vout, vin, sizeof(double) * 2 * (size_t)n);
    int totD = 0, totS = 0, corrCount = 0;
    double corrAcc = 0.0, corrMax = 0.0;
    for (int iz = 0; iz < nz; ++iz) {
        oracle_cell_ids(p, xout, cid);
        memset(cnt, 0, sizeof(int32_t) * (size_t)Nc);
        for (int i = 0; i < n; ++i) cnt[cid[i]]++;
        for (int c = 0; c < Nc; ++c) start[c + 1] = start[c] + cnt[c];
        memcpy(cur, start, sizeof(int32_t) * (size_t)Nc);
        for (int i = 0; i < n; ++i) ids[cur[cid[i]]++] = i;
        memcpy(vsnap, vout, sizeof(double) * 2 * (size_t)n);
        int mD = 0, mS = 0;
        double s4 = 0.0, s5 = 0.0;
        zone_kernel(p, zones[iz], cnt, start, ids, vsnap, xout, vout, seedBase + 104729ULL * (uint64_t)(iz + 1), &mD, &mS,
                    &s4, &s5);
        totD += mD;
        totS += mS;
        if (s4 > 0.0) { corrAcc += s4 * s4; ++corrCount; }
        corrMax = dmax(corrMax, s5);
    }
    if (m) {
        memset(m, 0, sizeof *m);
        m->nZones = nz;
        m->nThreadsRequested = 1;
        m->nThreadsUsed = 1;
        m->nParticlesMovedDense = totD;
        m->nParticlesMovedSparse = totS;
        m->corrRmsDU = (corrCount > 0) ? sqrt(corrAcc / (double)corrCount) : 0.0;
        m->corrMaxDU = corrMax;
    }
    free(cid); free(cnt); free(start); free(cur); free(ids); free(owner); free(vsnap); free(zones);
    return MPCD_OK;
}

/* ============================================================== liquid closure */

static double rho_target(const P* p) {
    const double Vc = (p->Lx / (double)p->Nx) * (p->Ly / (double)p->Ny);
    return p->gamma / Vc;
}

/* boundary_mask_from_owner (src/liquid_closure.cpp:143-160) */
static void boundary_mask(const P* p, const int32_t* own, int32_t* mask) {
    for (int ix = 0; ix < p->Nx; ++ix)
        for (int iy = 0; iy < p->Ny; ++iy) {
            const int c = iy + p->Ny * ix;
            const int right = (ix + 1 < p->Nx) ? iy + p->Ny * (ix + 1) : (periodic_x(p) ? iy : -1);
            const int up = (iy + 1 < p->Ny) ? (iy + 1) + p->Ny * ix : (periodic_y(p) ? p->Ny * ix : -1);
            int b = 0;
            if (right >= 0 && own[right] != own[c]) b = 1;
            if (up >= 0 && own[up] != own[c]) b = 1;
            mask[c] = b;
        }
}

/* dilate_mask (src/liquid_closure.cpp:162-195) */
static void dilate(const P* p, const int32_t* in, int32_t* out, int w) {
    if (w <= 0) { memcpy(out, in, sizeof(int32_t) * (size_t)p->Nc); return; }
    for (int ix = 0; ix < p->Nx; ++ix)
        for (int iy = 0; iy < p->Ny; ++iy) {
            int on = 0;
            for (int dx = -w; dx <= w && !on; ++dx)
                for (int dy = -w; dy <= w; ++dy) {
                    int jx = ix + dx, jy = iy + dy;
                    if (periodic_x(p)) jx = wrap_index(jx, p->Nx);
                    else if (jx < 0 || jx >= p->Nx) continue;
                    if (periodic_y(p)) jy = wrap_index(jy, p->Ny);
                    else if (jy < 0 || jy >= p->Ny) continue;
                    if (in[jy + p->Ny * jx] != 0) { on = 1; break; }
                }
            out[iy + p->Ny * ix] = on;
        }
}

/* build_interzone_mask (src/liquid_closure.cpp:197-213) */
void oracle_interzone_mask(const P* p, int32_t* mask) {
    const int Nc = p->Nc;
    memset(mask, 0, sizeof(int32_t) * (size_t)Nc);
    if (!p->smoothPdriveAtInterzone || !p->useZoneRedistribution || p->zonePassthroughMode || p->zoneSingleFullDomainMode) return;
    int32_t* own = (int32_t*)malloc(sizeof(int32_t) * (size_t)Nc);
    int32_t* b = (int32_t*)malloc(sizeof(int32_t) * (size_t)Nc);
    oracle_zone_owner_map(p, MPCD_LAYOUT_BASE, own);
    boundary_mask(p, own, b);
    dilate(p, b, mask, p->smoothPdriveInterzoneWidthCells);
    if (p->smoothPdriveIncludeShiftedLayouts) {
        int32_t* s = (int32_t*)malloc(sizeof(int32_t) * (size_t)Nc);
        oracle_zone_owner_map(p, MPCD_LAYOUT_SHIFTED, own);
        boundary_mask(p, own, b);
        dilate(p, b, s, p->smoothPdriveInterzoneWidthCells);
        for (int c = 0; c < Nc; ++c) mask[c] = (mask[c] || s[c]) ? 1 : 0;
        free(s);
    }
    free(own); free(b);
}

/* apply_cell_kick (src/liquid_closure.cpp:302-325) */
static void cell_kick(const P* p, double* v, const int32_t* cid, const double* kx, const double* ky, double* rms, double* mx) {
    double acc = 0.0, m = 0.0;
    for (int i = 0; i < p->n; ++i) {
        const int c = cid[i];
        v[2 * i] += kx[c];
        v[2 * i + 1] += ky[c];
        const double kn = sqrt(kx[c] * kx[c] + ky[c] * ky[c]);
        acc += kn * kn;
        if (kn > m) m = kn;
    }
    *rms = (p->n > 0) ? sqrt(acc / (double)p->n) : 0.0;
    *mx = (p->n > 0) ? m : 0.0;
}

static void fields_alloc(mpcd_cellfields_c* G, int Nc, double* buf, int32_t* nbuf) {
    G->N = nbuf;
    double** d[10] = {&G->Ux, &G->Uy, &G->Px, &G->Py, &G->T, &G->rho, &G->Pkin, &G->Pvir, &G->P, &G->rhoTarget};
    for (int k = 0; k < 10; ++k) *d[k] = buf + (size_t)k * Nc;
}

static void fields_copy(const mpcd_cellfields_c* src, mpcd_cellfields_c* dst, int Nc) {
    if (dst->N) memcpy(dst->N, src->N, sizeof(int32_t) * (size_t)Nc);
    double* s[10] = {src->Ux, src->Uy, src->Px, src->Py, src->T, src->rho, src->Pkin, src->Pvir, src->P, src->rhoTarget};
    double* d[10] = {dst->Ux, dst->Uy, dst->Px, dst->Py, dst->T, dst->rho, dst->Pkin, dst->Pvir, dst->P, dst->rhoTarget};
    for (int k = 0; k < 10; ++k) if (d[k]) memcpy(d[k], s[k], sizeof(double) * (size_t)Nc);
}

/* run_liquid_closure (src/liquid_closure.cpp:329-444) */
int oracle_liquid_closure(const P* p, const double* refx, const double* refv, const double* redx, const double* redv,
                          double* outx, double* outv, mpcd_closure_metrics_c* M, mpcd_closure_detail_c* D) {
    if (!p->useLiquidClosure) return fail(MPCD_ERR_INVALID_ARG, "run_liquid_closure requires useLiquidClosure=true");
    const int n = p->n, Nc = p->Nc;
    const double rhoT = rho_target(p);
    double* fb = (double*)calloc(40 * (size_t)Nc, sizeof(double));
    int32_t* nb = (int32_t*)calloc(4 * (size_t)Nc, sizeof(int32_t));
    mpcd_cellfields_c ref, red, rep, out;
    fields_alloc(&ref, Nc, fb, nb);
    fields_alloc(&red, Nc, fb + 10 * (size_t)Nc, nb + Nc);
    fields_alloc(&rep, Nc, fb + 20 * (size_t)Nc, nb + 2 * (size_t)Nc);
    fields_alloc(&out, Nc, fb + 30 * (size_t)Nc, nb + 3 * (size_t)Nc);
    oracle_cell_fields(p, refx, refv, rhoT, &ref);
    oracle_cell_fields(p, redx, redv, rhoT, &red);
    double* g = (double*)calloc(8 * (size_t)Nc, sizeof(double));
    double *duRX = g, *duRY = g + Nc, *appX = g + 2 * Nc, *appY = g + 3 * Nc, *praw = g + 4 * Nc, *pdr = g + 5 * Nc,
           *eosX = g + 6 * Nc, *eosY = g + 7 * Nc;
    mpcd_closure_metrics_c m;
    memset(&m, 0, sizeof m);
    double num = 0.0, den = 0.0;
    for (int c = 0; c < Nc; ++c) {
        duRX[c] = (ref.Px[c] - red.Px[c]) / p->gamma;
        duRY[c] = (ref.Py[c] - red.Py[c]) / p->gamma;
        const double ex = red.Ux[c] - ref.Ux[c], ey = red.Uy[c] - ref.Uy[c];
        num += -(ex * duRX[c] + ey * duRY[c]);
        den += duRX[c] * duRX[c] + duRY[c] * duRY[c];
    }
    m.betaRepairNum = num;
    m.betaRepairDen = den;
    double opt = 0.0;
    if (isfinite(num) && isfinite(den) && den > 0.0) opt = dmax(num / den, 0.0);
    m.betaRepairOpt = opt;
    if (!p->useOptimalBetaRepair) m.betaRepairApplied = p->betaRepair;
    else if (!isfinite(opt) || !isfinite(den) || den < 1e-20) m.betaRepairApplied = p->betaRepair;
    else m.betaRepairApplied = (opt < 0.0) ? 0.0 : ((2.0 < opt) ? 2.0 : opt);
    m.betaEOSApplied = p->betaEOS;
    double* rx = (double*)malloc(sizeof(double) * 2 * (size_t)(n > 0 ? n : 1));
    double* rv = (double*)malloc(sizeof(double) * 2 * (size_t)(n > 0 ? n : 1));
    memcpy(rx, redx, sizeof(double) * 2 * (size_t)n);
    memcpy(rv, redv, sizeof(double) * 2 * (size_t)n);
    int32_t* cidR = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    oracle_cell_ids(p, redx, cidR);
    for (int c = 0; c < Nc; ++c) { appX[c] = m.betaRepairApplied * duRX[c]; appY[c] = m.betaRepairApplied * duRY[c]; }
    cell_kick(p, rv, cidR, appX, appY, &m.rmsRepairDU, &m.maxRepairDU);
    double accAbs = 0.0;
    for (int c = 0; c < Nc; ++c) accAbs += hypot(appX[c], appY[c]);
    m.meanAbsRepairDU = accAbs / (double)imax(Nc, 1);
    oracle_cell_fields(p, rx, rv, rhoT, &rep);
    double s = 0.0;
    for (int c = 0; c < Nc; ++c) { praw[c] = ref.Pkin[c] + ref.Pvir[c]; s += praw[c]; }
    m.meanPdriveRaw = (Nc > 0) ? s / (double)Nc : 0.0;
    memcpy(pdr, praw, sizeof(double) * (size_t)Nc);
    int32_t* mask = (int32_t*)malloc(sizeof(int32_t) * (size_t)Nc);
    oracle_interzone_mask(p, mask);
    int nmask = 0;
    for (int c = 0; c < Nc; ++c) nmask += (mask[c] == 1);
    m.nMaskedInterzoneCells = nmask;
    if (nmask > 0) {
        /* local_cross_smooth (src/liquid_closure.cpp:215-241) */
        for (int ix = 0; ix < p->Nx; ++ix)
            for (int iy = 0; iy < p->Ny; ++iy) {
                const int c = iy + p->Ny * ix;
                if (mask[c] == 0) continue;
                double acc = praw[c];
                int k = 1;
                const int jj[4][2] = {{iy, ix - 1}, {iy, ix + 1}, {iy - 1, ix}, {iy + 1, ix}};
                for (int q = 0; q < 4; ++q) {
                    int jy = jj[q][0], jx = jj[q][1];
                    if (periodic_x(p)) jx = wrap_index(jx, p->Nx);
                    else if (jx < 0 || jx >= p->Nx) continue;
                    if (periodic_y(p)) jy = wrap_index(jy, p->Ny);
                    else if (jy < 0 || jy >= p->Ny) continue;
                    acc += praw[jy + p->Ny * jx];
                    ++k;
                }
                const double ps = acc / (double)k;
                pdr[c] = (1.0 - p->smoothPdriveInterzoneBlend) * praw[c] + p->smoothPdriveInterzoneBlend * ps;
            }
    }
    s = 0.0;
    for (int c = 0; c < Nc; ++c) s += pdr[c];
    m.meanPdrive = (Nc > 0) ? s / (double)Nc : 0.0;
    /* gradient_boundary_aware (src/liquid_closure.cpp:243-295) and the EOS kick (:424-430) */
    const double dx = p->Lx / (double)p->Nx, dy = p->Ly / (double)p->Ny;
    for (int ix = 0; ix < p->Nx; ++ix)
        for (int iy = 0; iy < p->Ny; ++iy) {
            const int c = iy + p->Ny * ix;
            double gx, gy;
            if (periodic_x(p)) gx = (pdr[iy + p->Ny * wrap_index(ix + 1, p->Nx)] - pdr[iy + p->Ny * wrap_index(ix - 1, p->Nx)]) / (2.0 * dx);
            else if (ix == 0) gx = (pdr[iy + p->Ny * (ix + 1)] - pdr[c]) / dx;
            else if (ix == p->Nx - 1) gx = (pdr[c] - pdr[iy + p->Ny * (ix - 1)]) / dx;
            else gx = (pdr[iy + p->Ny * (ix + 1)] - pdr[iy + p->Ny * (ix - 1)]) / (2.0 * dx);
            if (periodic_y(p)) gy = (pdr[wrap_index(iy + 1, p->Ny) + p->Ny * ix] - pdr[wrap_index(iy - 1, p->Ny) + p->Ny * ix]) / (2.0 * dy);
            else if (iy == 0) gy = (pdr[(iy + 1) + p->Ny * ix] - pdr[c]) / dy;
            else if (iy == p->Ny - 1) gy = (pdr[c] - pdr[(iy - 1) + p->Ny * ix]) / dy;
            else gy = (pdr[(iy + 1) + p->Ny * ix] - pdr[(iy - 1) + p->Ny * ix]) / (2.0 * dy);
            eosX[c] = -(p->dt / rhoT) * gx * p->betaEOS;
            eosY[c] = -(p->dt / rhoT) * gy * p->betaEOS;
        }
    memcpy(outx, rx, sizeof(double) * 2 * (size_t)n);
    memcpy(outv, rv, sizeof(double) * 2 * (size_t)n);
    cell_kick(p, outv, cidR, eosX, eosY, &m.rmsEOSDU, &m.maxEOSDU);
    oracle_cell_fields(p, outx, outv, rhoT, &out);
    double pix = 0.0, piy = 0.0, pox = 0.0, poy = 0.0;
    for (int i = 0; i < n; ++i) { pix += redv[2 * i]; piy += redv[2 * i + 1]; }
    for (int i = 0; i < n; ++i) { pox += outv[2 * i]; poy += outv[2 * i + 1]; }
    m.momentumDeltaX = pox - pix;
    m.momentumDeltaY = poy - piy;
    if (M) *M = m;
    if (D) {
        if (D->repairedX) memcpy(D->repairedX, rx, sizeof(double) * 2 * (size_t)n);
        if (D->repairedV) memcpy(D->repairedV, rv, sizeof(double) * 2 * (size_t)n);
        fields_copy(&ref, &D->refFields, Nc);
        fields_copy(&red, &D->redFields, Nc);
        fields_copy(&rep, &D->repairedFields, Nc);
        fields_copy(&out, &D->outFields, Nc);
        double* src[6] = {praw, pdr, duRX, duRY, eosX, eosY};
        double* dst[6] = {D->pdriveRaw, D->pdrive, D->duRepairX, D->duRepairY, D->duEOSX, D->duEOSY};
        for (int k = 0; k < 6; ++k) if (dst[k]) memcpy(dst[k], src[k], sizeof(double) * (size_t)Nc);
        if (D->interzoneMask) memcpy(D->interzoneMask, mask, sizeof(int32_t) * (size_t)Nc);
    }
    free(fb); free(nb); free(g); free(rx); free(rv); free(cidR); free(mask);
    return MPCD_OK;
}

/* ==================================================================== full step */

static void occstd_outband(const P* p, const int32_t* N, double* occ, double* ob) {
    double highThr, lowThr;
    thresholds(p, &highThr, &lowThr);
    int outc = 0;
    double mean = 0.0, var = 0.0;
    for (int c = 0; c < p->Nc; ++c) {
        const double n = (double)N[c];
        if ((n > highThr) || (n > 0.0 && n < lowThr)) ++outc;
        mean += n;
    }
    mean /= imax(1, p->Nc);
    for (int c = 0; c < p->Nc; ++c) { const double d = (double)N[c] - mean; var += d * d; }
    var /= imax(1, p->Nc);
    *occ = sqrt(var) / dmax(p->gamma, 1e-12);
    *ob = (double)outc / imax(1, p->Nc);
}

/* One iteration of the profiled benchmark loop (reference
 * main_benchmark_poiseuille_openmp_profiled_shifted_profiled.cpp:241-279) plus its metrics
 * row (:288-336). x, v are updated in place. */
int oracle_step(const P* p, double* x, double* v, int64_t step, mpcd_step_metrics_c* M) {
    const int n = p->n, Nc = p->Nc;
    const uint64_t s = (uint64_t)step;
    const size_t sz = sizeof(double) * 2 * (size_t)(n > 0 ? n : 1);
    double *rx = (double*)malloc(sz), *rv = (double*)malloc(sz), *bx = (double*)malloc(sz), *bv = (double*)malloc(sz),
           *sx = (double*)malloc(sz), *sv = (double*)malloc(sz);
    int32_t* cid = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    memcpy(rx, x, sizeof(double) * 2 * (size_t)n);
    memcpy(rv, v, sizeof(double) * 2 * (size_t)n);
    mpcd_step_metrics_c m;
    memset(&m, 0, sizeof m);
    m.step = step;
    int rc = MPCD_OK;
    oracle_stream(p, rx, rv);
    rc = oracle_apply_bc(p, rx, rv, 104729ULL + 10007ULL * s, &m.wall);
    if (!rc) {
        oracle_srd_shift_cells(p, rx, 130363ULL + 10007ULL * s, cid);
        rc = oracle_srd_collide(p, rv, cid, 433494437ULL + 10007ULL * s);
    }
    if (!rc) rc = oracle_zone_pass(p, rx, rv, bx, bv, MPCD_LAYOUT_BASE, 88172645463325252ULL + 10007ULL * s, &m.base);
    if (!rc) rc = oracle_zone_pass(p, bx, bv, sx, sv, MPCD_LAYOUT_SHIFTED, 88172645463325252ULL + 4099ULL + 10007ULL * s, &m.shifted);
    if (!rc) {
        mpcd_closure_detail_c D;
        memset(&D, 0, sizeof D);
        double* ofb = (double*)calloc(2 * (size_t)Nc, sizeof(double));
        D.outFields.Ux = ofb;
        D.outFields.Uy = ofb + Nc;
        rc = oracle_liquid_closure(p, rx, rv, sx, sv, x, v, &m.closure, &D);
        if (!rc && M) {
            int32_t* N = (int32_t*)calloc((size_t)Nc, sizeof(int32_t));
            oracle_cell_ids(p, bx, cid);
            for (int i = 0; i < n; ++i) N[cid[i]]++;
            occstd_outband(p, N, &m.baseOccStd, &m.baseOutBand);
            memset(N, 0, sizeof(int32_t) * (size_t)Nc);
            oracle_cell_ids(p, sx, cid);
            for (int i = 0; i < n; ++i) N[cid[i]]++;
            occstd_outband(p, N, &m.shiftedOccStd, &m.shiftedOutBand);
            m.occStd = m.shiftedOccStd;
            m.outBand = m.shiftedOutBand;
            double ke = 0.0, mx = 0.0, my = 0.0, su = 0.0, sw = 0.0;
            for (int i = 0; i < n; ++i) ke += 0.5 * (v[2 * i] * v[2 * i] + v[2 * i + 1] * v[2 * i + 1]);
            for (int i = 0; i < n; ++i) mx += v[2 * i];
            for (int i = 0; i < n; ++i) my += v[2 * i + 1];
            const double nn = (double)imax(n, 1);
            m.meanKinetic = ke / nn;
            m.meanVelocityX = mx / nn;
            m.meanVelocityY = my / nn;
            for (int c = 0; c < Nc; ++c) su += ofb[c];
            for (int c = 0; c < Nc; ++c) sw += ofb[Nc + c];
            m.meanUx = (Nc > 0) ? su / (double)Nc : 0.0;
            m.meanUy = (Nc > 0) ? sw / (double)Nc : 0.0;
            m.Qx = m.meanUx * p->Ly;
            free(N);
        }
        free(ofb);
    }
    if (M && !rc) *M = m;
    free(rx); free(rv); free(bx); free(bv); free(sx); free(sv); free(cid);
    return rc;
}

int oracle_run(const P* p, double* x, double* v, int64_t step0, int64_t nsteps, mpcd_step_metrics_c* last) {
    for (int64_t k = 1; k <= nsteps; ++k) {
        const int rc = oracle_step(p, x, v, step0 + k, (k == nsteps) ? last : NULL);
        if (rc) return rc;
    }
    return MPCD_OK;
}

/* hypot/atan2 used by the device tables: exported so tests can check them against glibc */
double oracle_log(double x) { return log(x); }
double oracle_hypot(double a, double b) { return hypot(a, b); }
