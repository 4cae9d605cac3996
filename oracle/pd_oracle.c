/*
 * pd_oracle.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * FP64 CPU restatement of the Peridynamics.jl explicit-dynamics hot path. Every function
 * cites the reference file:line it restates. The arithmetic keeps Julia's evaluation order
 * (left-associative products, StaticArrays' unrolled sums, no FMA contraction) so that an
 * FP64 GPU path that uses the same order can be compared bit for bit where the summation
 * order agrees.
 *
 * The force loop keeps the reference's serial scatter semantics (b_j -= p V_i while point i
 * is processed) for n_chunks == 1. With n_chunks > 1 it follows the threads backend of the
 * reference (src/core/threads_body_data_handler.jl:184-195): points are split into equal
 * index ranges, every chunk scatters into its own force buffer and the halo contributions
 * are added to the owning rows afterwards (src/core/halo_exchange.jl), which changes only
 * the summation order.
 *
 * Build: see oracle/Makefile (gcc -O2 -ffp-contract=off -fopenmp).
 */
#include "pd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int g_threads = 1;
static int g_serial_order = 0;

void or_set_threads(int32_t n) { g_threads = n < 1 ? 1 : n; }

/* 1: the state-based force loops keep the serial loop's summation order on every thread
 * count (or_force_density's serial-order gather); 0: the threads backend's chunked scatter */
void or_set_serial_order(int32_t on) { g_serial_order = on != 0; }

/* ------------------------------------------------------------------------------------ */
/* small 3-vector / 3x3 helpers in the order StaticArrays.jl unrolls them                */
/* matrices are column-major: A[r + 3c]                                                  */
/* ------------------------------------------------------------------------------------ */

static inline double dot3(const double *a, const double *b) {
    return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
}

static inline void cross3(const double *a, const double *b, double *c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

/* StaticArrays 3x3 det: vecdot(col1, cross(col2, col3)) */
double or_det3(const double *A) {
    double c[3];
    cross3(A + 3, A + 6, c);
    return dot3(A, c);
}

/* StaticArrays 3x3 inv (cross-product form): rows of the inverse are the cross products of
 * the columns divided by the determinant. */
void or_inv3(const double *A, double *R) {
    double x0[3] = {A[0], A[1], A[2]};
    const double *x1 = A + 3, *x2 = A + 6;
    double y0[3], y1[3], y2[3];
    cross3(x1, x2, y0);
    double d = dot3(x0, y0);
    for (int k = 0; k < 3; k++) { x0[k] = x0[k] / d; y0[k] = y0[k] / d; }
    cross3(x2, x0, y1);
    cross3(x0, x1, y2);
    /* column-major result (y0[1], y1[1], y2[1], y0[2], ...) */
    for (int c = 0; c < 3; c++) { R[0 + 3 * c] = y0[c]; R[1 + 3 * c] = y1[c]; R[2 + 3 * c] = y2[c]; }
}

/* C = A * B, entries summed k = 1..3 left to right */
static inline void matmul3(const double *A, const double *B, double *C) {
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++)
            C[r + 3 * c] = (A[r + 0] * B[0 + 3 * c] + A[r + 3] * B[1 + 3 * c]) + A[r + 6] * B[2 + 3 * c];
}

/* C = A' * B */
static inline void matTmul3(const double *A, const double *B, double *C) {
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++)
            C[r + 3 * c] = (A[0 + 3 * r] * B[0 + 3 * c] + A[1 + 3 * r] * B[1 + 3 * c]) + A[2 + 3 * r] * B[2 + 3 * c];
}

/* C = A * B' */
static inline void matmulT3(const double *A, const double *B, double *C) {
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++)
            C[r + 3 * c] = (A[r + 0] * B[c + 0] + A[r + 3] * B[c + 3]) + A[r + 6] * B[c + 6];
}

static inline void matvec3(const double *A, const double *v, double *w) {
    for (int r = 0; r < 3; r++) w[r] = (A[r] * v[0] + A[r + 3] * v[1]) + A[r + 6] * v[2];
}

static inline int has_nan9(const double *A) {
    for (int k = 0; k < 9; k++) if (isnan(A[k])) return 1;
    return 0;
}

/* Julia: Bool * Float64 = ifelse(b, x, copysign(0, x)) */
static inline double bmul(int b, double x) { return b ? x : copysign(0.0, x); }

/* ------------------------------------------------------------------------------------ */
/* material parameters: src/physics/material_parameters.jl:118-231, fracture.jl:110-130,  */
/* bond_based.jl:86-113, correspondence.jl:163-169                                       */
/* ------------------------------------------------------------------------------------ */
int or_point_params(int32_t material, double delta, double rho, double E, double nu, double G,
                    double K, double lambda, double mu, double Gc, double epsc,
                    or_params *out, char *msg, int32_t msg_len) {
    /* E, nu, G, K, lambda, mu: NaN when not given; Gc, epsc: NaN when not given */
    if (!(delta > 0)) { snprintf(msg, msg_len, "`horizon` should be larger than zero!"); return 1; }
    if (!(rho > 0)) { snprintf(msg, msg_len, "`rho` should be larger than zero!"); return 1; }
    if (material == OR_BB) {
        /* bond_based.jl:93-103: nu must be 1/4; with a single elastic keyword, nu := 0.25 */
        int nfin = isfinite(E) + isfinite(nu) + isfinite(G) + isfinite(K) + isfinite(lambda) + isfinite(mu);
        if (isfinite(nu) && fabs(nu - 0.25) > 1.4901161193847656e-8 * fmax(fabs(nu), 0.25)) {
            snprintf(msg, msg_len, "Bond-based peridynamics has a limitation on the Poisson's ratio!"); return 1;
        }
        if (!isfinite(nu) && nfin == 1) nu = 0.25;
    }
    /* get_given_elastic_params + check_elastic_params */
    int nfin = isfinite(E) + isfinite(nu) + isfinite(G) + isfinite(K) + isfinite(lambda) + isfinite(mu);
    if (isfinite(G) && isfinite(mu)) { snprintf(msg, msg_len, "`G` and `mu` are defined!"); return 1; }
    if (nfin < 2) { snprintf(msg, msg_len, "Not enough material parameters defined!"); return 1; }
    if (nfin > 2) { snprintf(msg, msg_len, "Too many material parameters defined!"); return 1; }
    /* get_E_and_nu */
    if (isfinite(E) && isfinite(nu)) {
    } else if (isfinite(E) && isfinite(G)) { nu = E / (2 * G) - 1;
    } else if (isfinite(E) && isfinite(K)) { nu = (3 * K - E) / (6 * K);
    } else if (isfinite(E) && isfinite(lambda)) { nu = (-(E + lambda) + sqrt((E + lambda) * (E + lambda) + 8 * (lambda * lambda))) / (4 * lambda);
    } else if (isfinite(E) && isfinite(mu)) { nu = E / (2 * mu) - 1;
    } else if (isfinite(nu) && isfinite(G)) { E = 2 * G * (1 + nu);
    } else if (isfinite(nu) && isfinite(K)) { E = 3 * K * (1 - 2 * nu);
    } else if (isfinite(nu) && isfinite(lambda)) { E = (lambda * (1 + nu) * (1 - 2 * nu)) / nu;
    } else if (isfinite(nu) && isfinite(mu)) { E = 2 * mu * (1 + nu);
    } else if (isfinite(G) && isfinite(K)) { E = 9 * K * G / (3 * K + G); nu = (3 * K - 2 * G) / (2 * (3 * K + G));
    } else if (isfinite(G) && isfinite(lambda)) { E = G * (3 * lambda + 2 * G) / (lambda + G); nu = lambda / (2 * (lambda + G));
    } else if (isfinite(K) && isfinite(lambda)) { E = 9 * K * (K - lambda) / (3 * K - lambda); nu = lambda / (3 * K - lambda);
    } else if (isfinite(K) && isfinite(mu)) { E = 9 * K * mu / (3 * K + mu); nu = (3 * K - 2 * mu) / (2 * (3 * K + mu));
    } else if (isfinite(lambda) && isfinite(mu)) { E = mu * (3 * lambda + 2 * mu) / (lambda + mu); nu = lambda / (2 * (lambda + mu));
    }
    double Gm = E / (2 * (1 + nu));
    double Km = E / (3 * (1 - 2 * nu));
    double lam = E * nu / ((1 + nu) * (1 - 2 * nu));
    if (material == OR_BB && fabs(nu - 0.25) > 1.4901161193847656e-8 * fmax(fabs(nu), 0.25)) {
        snprintf(msg, msg_len, "Bond-based peridynamics has a limitation on the Poisson's ratio!"); return 1;
    }
    out->delta = delta; out->rho = rho; out->E = E; out->nu = nu; out->G = Gm; out->K = Km;
    out->lambda = lam; out->mu = Gm;
    /* fracture.jl:110-130 */
    if (isfinite(Gc) && !isfinite(epsc)) {
        out->Gc = Gc; out->epsc = sqrt(5.0 * Gc / (9.0 * Km * delta));
    } else if (!isfinite(Gc) && isfinite(epsc)) {
        out->epsc = epsc; out->Gc = 9.0 / 5.0 * Km * delta * (epsc * epsc);
    } else if (isfinite(Gc) && isfinite(epsc)) {
        snprintf(msg, msg_len, "Define either Gc or epsilon_c, not both!"); return 1;
    } else { out->Gc = 0.0; out->epsc = 0.0; }
    /* bc = 18 * K / (pi * delta^4), delta^4 by repeated squaring */
    double d2 = delta * delta;
    out->bc = 18 * Km / (M_PI * (d2 * d2));
    return 0;
}

/* ------------------------------------------------------------------------------------ */
/* bond search: src/discretization/bond_system.jl:96-165                                 */
/* all neighbours j != i with |X_j - X_i|^2 <= delta_i^2, ordered by ascending j (the    */
/* reference's order comes from PointNeighbors.foreach_neighbor and is not pinned for     */
/* large lattices; ascending j is this restatement's fixed choice). fail_permit of a bond */
/* is fp_i & fp_j. Filter-mode pre-cracks (precrack!(...; update_dmg=false)) delete the  */
/* bonds between the two point sets.                                                      */
/* ------------------------------------------------------------------------------------ */
static int cmp_i32(const void *a, const void *b) {
    int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    return (x > y) - (x < y);
}

typedef struct { int64_t nc[3]; double lo[3]; double h; int64_t *cell_start; int32_t *cell_pts; } grid_t;

static void grid_build(grid_t *g, int64_t n, const double *X, double h) {
    for (int d = 0; d < 3; d++) {
        double lo = INFINITY, hi = -INFINITY;
        for (int64_t i = 0; i < n; i++) { double x = X[3 * i + d]; if (x < lo) lo = x; if (x > hi) hi = x; }
        if (n == 0) { lo = 0; hi = 0; }
        g->lo[d] = lo;
        g->nc[d] = (int64_t)floor((hi - lo) / h) + 1;
        if (g->nc[d] < 1) g->nc[d] = 1;
    }
    g->h = h;
    int64_t ncell = g->nc[0] * g->nc[1] * g->nc[2];
    g->cell_start = (int64_t *)calloc((size_t)ncell + 1, sizeof(int64_t));
    g->cell_pts = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    int64_t *cid = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    for (int64_t i = 0; i < n; i++) {
        int64_t c[3];
        for (int d = 0; d < 3; d++) {
            c[d] = (int64_t)floor((X[3 * i + d] - g->lo[d]) / h);
            if (c[d] < 0) c[d] = 0;
            if (c[d] >= g->nc[d]) c[d] = g->nc[d] - 1;
        }
        cid[i] = c[0] + g->nc[0] * (c[1] + g->nc[1] * c[2]);
        g->cell_start[cid[i] + 1]++;
    }
    for (int64_t c = 0; c < ncell; c++) g->cell_start[c + 1] += g->cell_start[c];
    int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * (size_t)(ncell > 0 ? ncell : 1));
    memcpy(fill, g->cell_start, sizeof(int64_t) * (size_t)ncell);
    for (int64_t i = 0; i < n; i++) g->cell_pts[fill[cid[i]]++] = (int32_t)i;
    free(fill);
    free(cid);
}

static int64_t neighbours_of(const grid_t *g, int64_t n, const double *X, int64_t i, double delta,
                             int32_t *buf, int64_t bufcap, int *dup) {
    int64_t c[3];
    for (int d = 0; d < 3; d++) {
        c[d] = (int64_t)floor((X[3 * i + d] - g->lo[d]) / g->h);
        if (c[d] < 0) c[d] = 0;
        if (c[d] >= g->nc[d]) c[d] = g->nc[d] - 1;
    }
    /* cells within ceil(delta / h) layers (delta <= h unless per-point horizons differ) */
    int64_t r = (int64_t)ceil(delta / g->h);
    if (r < 1) r = 1;
    double r2 = delta * delta;
    int64_t cnt = 0;
    for (int64_t cz = c[2] - r; cz <= c[2] + r; cz++) {
        if (cz < 0 || cz >= g->nc[2]) continue;
        for (int64_t cy = c[1] - r; cy <= c[1] + r; cy++) {
            if (cy < 0 || cy >= g->nc[1]) continue;
            for (int64_t cx = c[0] - r; cx <= c[0] + r; cx++) {
                if (cx < 0 || cx >= g->nc[0]) continue;
                int64_t cell = cx + g->nc[0] * (cy + g->nc[1] * cz);
                for (int64_t k = g->cell_start[cell]; k < g->cell_start[cell + 1]; k++) {
                    int32_t j = g->cell_pts[k];
                    if (j == i) continue;
                    /* PointNeighbors: pos_diff = x_i - x_j, distance2 = dot, keep if <= r^2 */
                    double dd[3] = {X[3 * i] - X[3 * j], X[3 * i + 1] - X[3 * j + 1], X[3 * i + 2] - X[3 * j + 2]};
                    double d2 = dot3(dd, dd);
                    if (d2 <= r2) {
                        if (sqrt(d2) < 2.220446049250313e-16) *dup = 1; /* check_point_duplicates */
                        if (buf && cnt < bufcap) buf[cnt] = j;
                        cnt++;
                    }
                }
            }
        }
    }
    (void)n;
    return cnt;
}

int64_t or_find_bonds(int64_t n, const double *X, const double *delta, const uint8_t *fp_point,
                      const uint8_t *crack_a, const uint8_t *crack_b, int32_t n_cracks,
                      int64_t cap, int64_t *off, int32_t *nbr, double *L, uint8_t *fail_permit) {
    double dmax = 0;
    for (int64_t i = 0; i < n; i++) if (delta[i] > dmax) dmax = delta[i];
    if (n == 0) { if (off) off[0] = 0; return 0; }
    grid_t g;
    grid_build(&g, n, X, dmax);
    int64_t *cnt = (int64_t *)calloc((size_t)n, sizeof(int64_t));
    int dup_any = 0;
    int64_t maxc = 0;
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 1024) reduction(| : dup_any) reduction(max : maxc)
    for (int64_t i = 0; i < n; i++) {
        int dup = 0;
        int64_t c = neighbours_of(&g, n, X, i, delta[i], NULL, 0, &dup);
        cnt[i] = c;
        dup_any |= dup;
        if (c > maxc) maxc = c;
    }
    if (dup_any) { free(cnt); free(g.cell_start); free(g.cell_pts); return -1; }
    /* crack filter (bond_system.jl:142-165) on the candidate lists */
    int64_t total = 0;
    int64_t *kept = (int64_t *)calloc((size_t)n, sizeof(int64_t));
#pragma omp parallel num_threads(g_threads)
    {
        int32_t *buf = (int32_t *)malloc(sizeof(int32_t) * (size_t)(maxc > 0 ? maxc : 1));
#pragma omp for schedule(dynamic, 1024)
        for (int64_t i = 0; i < n; i++) {
            int dup = 0;
            int64_t c = neighbours_of(&g, n, X, i, delta[i], buf, maxc, &dup);
            int64_t k = 0;
            for (int64_t q = 0; q < c; q++) {
                int32_t j = buf[q];
                int del = 0;
                for (int32_t cr = 0; cr < n_cracks; cr++) {
                    const uint8_t *A = crack_a + (size_t)cr * n, *B = crack_b + (size_t)cr * n;
                    if ((A[i] && B[j]) || (B[i] && A[j])) del = 1;
                }
                if (!del) k++;
            }
            kept[i] = k;
        }
        free(buf);
    }
    for (int64_t i = 0; i < n; i++) total += kept[i];
    if (cap < total || off == NULL) {
        free(cnt); free(kept); free(g.cell_start); free(g.cell_pts);
        return total;
    }
    off[0] = 0;
    for (int64_t i = 0; i < n; i++) off[i + 1] = off[i] + kept[i];
#pragma omp parallel num_threads(g_threads)
    {
        int32_t *buf = (int32_t *)malloc(sizeof(int32_t) * (size_t)(maxc > 0 ? maxc : 1));
#pragma omp for schedule(dynamic, 1024)
        for (int64_t i = 0; i < n; i++) {
            int dup = 0;
            int64_t c = neighbours_of(&g, n, X, i, delta[i], buf, maxc, &dup);
            qsort(buf, (size_t)c, sizeof(int32_t), cmp_i32);
            int64_t o = off[i];
            for (int64_t q = 0; q < c; q++) {
                int32_t j = buf[q];
                int del = 0;
                for (int32_t cr = 0; cr < n_cracks; cr++) {
                    const uint8_t *A = crack_a + (size_t)cr * n, *B = crack_b + (size_t)cr * n;
                    if ((A[i] && B[j]) || (B[i] && A[j])) del = 1;
                }
                if (del) continue;
                double dd[3] = {X[3 * i] - X[3 * j], X[3 * i + 1] - X[3 * j + 1], X[3 * i + 2] - X[3 * j + 2]};
                nbr[o] = j;
                L[o] = sqrt(dot3(dd, dd));
                fail_permit[o] = (uint8_t)(fp_point[i] & fp_point[j]);
                o++;
            }
        }
        free(buf);
    }
    free(cnt); free(kept); free(g.cell_start); free(g.cell_pts);
    return total;
}

/* find_kernels: bond_system.jl:184-201 with kernels.jl:10-52 (horizon of the bond owner) */
void or_kernels(const or_sys *sys, int32_t kernel, double *omega) {
    for (int64_t i = 0; i < sys->n; i++) {
        double d = sys->params[sys->pid[i]].delta;
        for (int64_t b = sys->off[i]; b < sys->off[i + 1]; b++) {
            double Lb = sys->L[b], w;
            if (kernel == OR_KERNEL_CONST_ONE) w = 1.0;
            else if (kernel == OR_KERNEL_LINEAR) w = d / Lb;
            else {
                double xi = Lb / d;
                if (0 < xi && xi <= 0.5) w = 2.0 / 3.0 - 4 * (xi * xi) + 4 * (xi * xi * xi);
                else if (0.5 < xi && xi <= 1) w = 4.0 / 3.0 - 4 * xi + 4 * (xi * xi) - 4.0 / 3.0 * (xi * xi * xi);
                else w = 0;
            }
            omega[b] = w;
        }
    }
}

/* storage initialisation: bond_system.jl:370-380, velocity_verlet.jl:342-352 */
void or_init_state(const or_sys *sys, or_state *st) {
    int64_t n = sys->n;
    memcpy(st->pos, sys->X, sizeof(double) * 3 * (size_t)n);
    memset(st->u, 0, sizeof(double) * 3 * (size_t)n);
    memset(st->v, 0, sizeof(double) * 3 * (size_t)n);
    memset(st->vh, 0, sizeof(double) * 3 * (size_t)n);
    memset(st->a, 0, sizeof(double) * 3 * (size_t)n);
    memset(st->b_int, 0, sizeof(double) * 3 * (size_t)n);
    memset(st->b_ext, 0, sizeof(double) * 3 * (size_t)n);
    for (int64_t i = 0; i < n; i++) { st->damage[i] = 0; st->n_active[i] = sys->off[i + 1] - sys->off[i]; }
    memset(st->bond_active, 1, (size_t)sys->n_bonds);
    if (st->bond_length) memset(st->bond_length, 0, sizeof(double) * (size_t)sys->n_bonds);
    if (st->defgrad) memset(st->defgrad, 0, sizeof(double) * 9 * (size_t)n);
    if (st->cauchy) memset(st->cauchy, 0, sizeof(double) * 9 * (size_t)n);
}

/* break_bonds!: bond_system.jl:249-267 */
void or_break_bonds(const or_sys *sys, or_state *st, const uint8_t *A, const uint8_t *B) {
    for (int64_t i = 0; i < sys->n; i++) {
        st->n_active[i] = 0;
        for (int64_t b = sys->off[i]; b < sys->off[i + 1]; b++) {
            int32_t j = sys->nbr[b];
            if ((A[i] && B[j]) || (B[i] && A[j])) st->bond_active[b] = 0;
            st->n_active[i] += st->bond_active[b];
        }
    }
}

/* calc_damage!: bond_system.jl:338-343 */
static inline void damage_point(const or_sys *sys, or_state *st, int64_t i) {
    int64_t nn = sys->off[i + 1] - sys->off[i];
    st->damage[i] = 1.0 - (double)st->n_active[i] / (double)nn;
}

void or_calc_damage(const or_sys *sys, or_state *st) {
    for (int64_t i = 0; i < sys->n; i++) damage_point(sys, st, i);
}

static inline const or_params *P_of(const or_sys *sys, int64_t i) { return &sys->params[sys->pid[i]]; }

/* surface_correction_factor (bond_system_corrections.jl:37-39, 72-75) */
#define SCF(sys, b) ((sys)->scfactor ? (sys)->scfactor[b] : 1.0)

/* calc_failure!: bond_system.jl:309-327 (generic) and bond_based.jl:125-144 /
 * ordinary_state_based.jl:107-126 (store the current bond length) */
static void failure_point(const or_sys *sys, or_state *st, int64_t i) {
    double epsc = P_of(sys, i)->epsc;
    const double *x = st->pos;
    int64_t na = 0;
    for (int64_t b = sys->off[i]; b < sys->off[i + 1]; b++) {
        int32_t j = sys->nbr[b];
        double Lb = sys->L[b];
        double d[3] = {x[3 * j] - x[3 * i], x[3 * j + 1] - x[3 * i + 1], x[3 * j + 2] - x[3 * i + 2]};
        double l = sqrt(dot3(d, d));
        double eps = (l - Lb) / Lb;
        if (st->bond_length) st->bond_length[b] = l;
        if (eps > epsc && sys->fail_permit[b]) st->bond_active[b] = 0;
        na += st->bond_active[b];
    }
    st->n_active[i] = na;
}

/* BB force_density_point!: bond_based.jl:146-180 */
static void bb_force_point(const or_sys *sys, or_state *st, int64_t i) {
    const double *x = st->pos;
    const or_params *pi = P_of(sys, i);
    double *bi = st->b_int + 3 * i;
    for (int64_t b = sys->off[i]; b < sys->off[i + 1]; b++) {
        int32_t j = sys->nbr[b];
        double Lb = sys->L[b];
        double d[3] = {x[3 * j] - x[3 * i], x[3 * j + 1] - x[3 * i + 1], x[3 * j + 2] - x[3 * i + 2]};
        double l = st->bond_length[b];
        double eps = (l - Lb) / Lb;
        double om = bmul(st->bond_active[b], SCF(sys, b));
        double s;
        if (sys->multi) s = om * (pi->bc + P_of(sys, j)->bc) / 2 * eps * sys->vol[j];
        else s = om * pi->bc * eps * sys->vol[j];
        for (int k = 0; k < 3; k++) bi[k] += s * d[k] / l;
    }
}

/* OSB: ordinary_state_based.jl:128-204 */
static void osb_force_point(const or_sys *sys, or_state *st, double *bsink, int64_t i) {
    const double *x = st->pos, *X = sys->X;
    const or_params *pi = P_of(sys, i);
    double wvol = 0.0;
    for (int64_t b = sys->off[i]; b < sys->off[i + 1]; b++) {
        int32_t j = sys->nbr[b];
        double D[3] = {X[3 * j] - X[3 * i], X[3 * j + 1] - X[3 * i + 1], X[3 * j + 2] - X[3 * i + 2]};
        double om = sys->omega[b] * (st->bond_active[b] ? 1.0 : 0.0);
        wvol += om * SCF(sys, b) * dot3(D, D) * sys->vol[j];
    }
    if (wvol == 0.0) return;
    double dil = 0.0, c1d = 3.0 / wvol;
    for (int64_t b = sys->off[i]; b < sys->off[i + 1]; b++) {
        int32_t j = sys->nbr[b];
        double Lb = sys->L[b], l = st->bond_length[b];
        double om = sys->omega[b] * (st->bond_active[b] ? 1.0 : 0.0);
        dil += om * SCF(sys, b) * c1d * Lb * (l - Lb) * sys->vol[j];
    }
    double c1 = 0, c2 = 0;
    if (!sys->multi) {
        c1 = 15.0 * pi->G / wvol;
        c2 = dil * (3.0 * pi->K / wvol - c1 / 3.0);
    }
    for (int64_t b = sys->off[i]; b < sys->off[i + 1]; b++) {
        int32_t j = sys->nbr[b];
        double Lb = sys->L[b], l = st->bond_length[b];
        double d[3] = {x[3 * j] - x[3 * i], x[3 * j + 1] - x[3 * i + 1], x[3 * j + 2] - x[3 * i + 2]};
        if (sys->multi) {
            const or_params *pj = P_of(sys, j);
            c1 = 15.0 * (pi->G + pj->G) / (2 * wvol);
            c2 = dil * (3.0 * (pi->K + pj->K) / (2 * wvol) - c1 / 3.0);
        }
        double om = sys->omega[b] * (st->bond_active[b] ? 1.0 : 0.0);
        double s = om * SCF(sys, b) * (c2 * Lb + c1 * (l - Lb)) / l;
        for (int k = 0; k < 3; k++) {
            double p = s * d[k];
            bsink[3 * i + k] += p * sys->vol[j];
            bsink[3 * j + k] += -p * sys->vol[i];
        }
    }
}

/* first_piola_kirchhoff: constitutive_models.jl:35-41 (SVK), 169-176 (NeoHooke),
 * 233-244 (NeoHookePenalty) */
void or_first_piola_kirchhoff(int32_t cmodel, const or_params *p, const double *F, double *P) {
    double C[9], S[9];
    if (cmodel == OR_SVK) {
        double E[9];
        matTmul3(F, F, C);
        for (int k = 0; k < 9; k++) E[k] = 0.5 * (C[k] - ((k % 4) == 0 ? 1.0 : 0.0));
        double trE = (E[0] + E[4]) + E[8];
        /* lambda tr(E) I + 2 mu E: the uniform scaling adds to the diagonal only */
        double a = p->lambda * trE, m2 = 2 * p->mu;
        for (int k = 0; k < 9; k++) S[k] = (k % 4) == 0 ? m2 * E[k] + a : m2 * E[k];
    } else if (cmodel == OR_NEOHOOKE) {
        double J = or_det3(F), Ci[9];
        matTmul3(F, F, C);
        or_inv3(C, Ci);
        double lj = p->lambda * log(J);
        /* I - Cinv: -Cinv with 1 added on the diagonal */
        for (int k = 0; k < 9; k++) S[k] = p->mu * ((k % 4) == 0 ? -Ci[k] + 1.0 : -Ci[k]) + lj * Ci[k];
    } else {
        double J = or_det3(F);
        if (J < 2.220446049250313e-16 || isnan(J)) { for (int k = 0; k < 9; k++) P[k] = 0.0; return; }
        double Ci[9];
        matTmul3(F, F, C);
        or_inv3(C, Ci);
        double trC = (C[0] + C[4]) + C[8];
        double a = 1.0 / 3.0 * trC;
        double jp = pow(J, -2.0 / 3.0);
        double ij = 1.0 / J;
        double vol = p->K / 4 * (J * J - ij * ij);
        for (int k = 0; k < 9; k++)
            S[k] = p->G * ((k % 4) == 0 ? -(a * Ci[k]) + 1.0 : -(a * Ci[k])) * jp + vol * Ci[k];
    }
    matmul3(F, S, P);
}

/* Hooke tensor entry C[i,j,k,l] (0-based) as get_hooke_matrix builds it from the Voigt matrix
 * (constitutive_models.jl:107-133): Voigt index of (i,j) in the order (1,1), (2,2), (3,3),
 * (2,3), (1,3), (1,2); a = (1 - nu) lambda / nu on the diagonal of the normal block, lambda off
 * it, mu on the diagonal of the shear block, zero elsewhere. */
static int voigt_index(int i, int j) {
    if (i == j) return i;
    int m = i + j;  /* {1,2} -> 3, {0,2} -> 2, {0,1} -> 1 */
    return m == 3 ? 3 : (m == 2 ? 4 : 5);
}

static double hooke_entry(const or_params *p, double a, int i, int j, int k, int l) {
    int I = voigt_index(i, j), J = voigt_index(k, l);
    if (I < 3 && J < 3) return I == J ? a : p->lambda;
    if (I >= 3 && J >= 3) return I == J ? p->mu : 0.0;
    return 0.0;
}

/* calc_zem_stiffness_tensor (zem_stabilization.jl:32-42): C_1[i,j] = sum over k (outer) and l
 * (inner) of C[i,j,k,l] Kinv[k,l], every one of the 81 products summed as the reference does;
 * column-major 3x3 result. */
void or_zem_wan_stiffness(const or_params *p, const double *Kinv, double *C1) {
    double a = (1 - p->nu) * p->lambda / p->nu;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double sum = 0.0;
            for (int k = 0; k < 3; k++)
                for (int l = 0; l < 3; l++) sum += hooke_entry(p, a, i, j, k, l) * Kinv[k + 3 * l];
            C1[i + 3 * j] = sum;
        }
}

/* the stabilisation term of bond b (c_force_density!, correspondence.jl:226-279):
 * ZEMSilling (w beta) z with beta = Cs bc / delta, ZEMWan (w C_1) z */
static inline void zem_term(const or_sys *sys, const or_params *p, const double *C1, double om,
                            const double *z, double *tz) {
    if (sys->zem == OR_ZEM_WAN) {
        double W1[9];
        for (int k = 0; k < 9; k++) W1[k] = om * C1[k];
        matvec3(W1, z, tz);
    } else {
        double beta = sys->zem_cs * p->bc / p->delta;
        double ob = om * beta;
        for (int k = 0; k < 3; k++) tz[k] = ob * z[k];
    }
}

/* CMaterial: correspondence.jl:183-279, 288-298; stress.jl:112-116 */
static void c_force_point(const or_sys *sys, or_state *st, double *bsink, int64_t i) {
    const double *x = st->pos, *X = sys->X;
    const or_params *pi = P_of(sys, i);
    double K[9] = {0}, Ft[9] = {0};
    for (int64_t b = sys->off[i]; b < sys->off[i + 1]; b++) {
        int32_t j = sys->nbr[b];
        double D[3] = {X[3 * j] - X[3 * i], X[3 * j + 1] - X[3 * i + 1], X[3 * j + 2] - X[3 * i + 2]};
        double d[3] = {x[3 * j] - x[3 * i], x[3 * j + 1] - x[3 * i + 1], x[3 * j + 2] - x[3 * i + 2]};
        double om = sys->omega[b] * (st->bond_active[b] ? 1.0 : 0.0);
        double temp = om * sys->vol[j];
        for (int c = 0; c < 3; c++)
            for (int r = 0; r < 3; r++) {
                K[r + 3 * c] = K[r + 3 * c] + temp * (D[r] * D[c]);
                Ft[r + 3 * c] = Ft[r + 3 * c] + temp * (d[r] * D[c]);
            }
    }
    double Kinv[9], F[9];
    or_inv3(K, Kinv);
    matmul3(Ft, Kinv, F);
    memcpy(st->defgrad + 9 * i, F, sizeof(F));
    if (st->damage[i] > sys->maxdmg || has_nan9(F)) {
        for (int64_t b = sys->off[i]; b < sys->off[i + 1]; b++) st->bond_active[b] = 0;
        st->n_active[i] = 0;
        return;
    }
    double P[9], PKinv[9], PF[9];
    or_first_piola_kirchhoff(sys->cmodel, pi, F, P);
    matmul3(P, Kinv, PKinv);
    double J = or_det3(F), iJ = 1 / J, Ps[9];
    for (int k = 0; k < 9; k++) Ps[k] = iJ * P[k];
    matmulT3(Ps, F, PF);
    memcpy(st->cauchy + 9 * i, PF, sizeof(PF));
    double C1[9] = {0};
    if (sys->zem == OR_ZEM_WAN) or_zem_wan_stiffness(pi, Kinv, C1);
    for (int64_t b = sys->off[i]; b < sys->off[i + 1]; b++) {
        int32_t j = sys->nbr[b];
        double D[3] = {X[3 * j] - X[3 * i], X[3 * j + 1] - X[3 * i + 1], X[3 * j + 2] - X[3 * i + 2]};
        double d[3] = {x[3 * j] - x[3 * i], x[3 * j + 1] - x[3 * i + 1], x[3 * j + 2] - x[3 * i + 2]};
        double om = sys->omega[b] * (st->bond_active[b] ? 1.0 : 0.0);
        double FD[3], z[3], W[9], WD[3], tz[3];
        matvec3(F, D, FD);
        for (int k = 0; k < 3; k++) z[k] = d[k] - FD[k];
        zem_term(sys, pi, C1, om, z, tz);
        for (int k = 0; k < 9; k++) W[k] = om * PKinv[k];
        matvec3(W, D, WD);
        for (int k = 0; k < 3; k++) {
            double t = WD[k] + tz[k];
            bsink[3 * i + k] += t * sys->vol[j];
            bsink[3 * j + k] += -t * sys->vol[i];
        }
    }
}

/* ------------------------------------------------------------------------------------ */
/* The serial loop's arithmetic on many threads. In the serial loop of bond_system.jl:       */
/* 285-297 point i's force row receives, in this order: the scattered terms -p V_k of every  */
/* point k < i bonded to i (in increasing k, one term per k), its own terms p V_j (its bond   */
/* order), then the scattered terms of the points k > i. A point's failure test and damage    */
/* touch only its own bonds, and its force terms read only its own bonds, so the failure      */
/* tests of all points can run first, then every point's state (OSB: weighted volume,         */
/* dilatation, c1, c2; CMat: F, P K^-1 and the kill decision), then every force row gathered  */
/* in the serial order: bit for bit the serial loop, on any number of threads.               */
/* ------------------------------------------------------------------------------------ */

/* position of i in the sorted bond list of j (the bond j -> i), or -1 */
static int64_t reverse_bond(const or_sys *sys, int64_t j, int64_t i) {
    int64_t lo = sys->off[j], hi = sys->off[j + 1];
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (sys->nbr[mid] < i) lo = mid + 1; else hi = mid;
    }
    return (lo < sys->off[j + 1] && sys->nbr[lo] == i) ? lo : -1;
}

/* OSB point state: weighted volume, dilatation (ordinary_state_based.jl:176-204) */
static void osb_state_point(const or_sys *sys, const or_state *st, int64_t i, double *wd) {
    const double *X = sys->X;
    double wvol = 0.0;
    for (int64_t b = sys->off[i]; b < sys->off[i + 1]; b++) {
        int32_t j = sys->nbr[b];
        double D[3] = {X[3 * j] - X[3 * i], X[3 * j + 1] - X[3 * i + 1], X[3 * j + 2] - X[3 * i + 2]};
        double om = sys->omega[b] * (st->bond_active[b] ? 1.0 : 0.0);
        wvol += om * SCF(sys, b) * dot3(D, D) * sys->vol[j];
    }
    double dil = 0.0;
    if (wvol != 0.0) {
        double c1d = 3.0 / wvol;
        for (int64_t b = sys->off[i]; b < sys->off[i + 1]; b++) {
            int32_t j = sys->nbr[b];
            double Lb = sys->L[b], l = st->bond_length[b];
            double om = sys->omega[b] * (st->bond_active[b] ? 1.0 : 0.0);
            dil += om * SCF(sys, b) * c1d * Lb * (l - Lb) * sys->vol[j];
        }
    }
    wd[0] = wvol;
    wd[1] = dil;
}

/* c1, c2 of a point with one parameter set (ordinary_state_based.jl:135-136), stored beside
 * its weighted volume and dilatation: wd = {wvol, dil, c1, c2} per point */
static void osb_coeffs_point(const or_sys *sys, int64_t i, double *wd) {
    const or_params *pi = P_of(sys, i);
    wd[2] = 0.0;
    wd[3] = 0.0;
    if (wd[0] != 0.0 && !sys->multi) {
        wd[2] = 15.0 * pi->G / wd[0];
        wd[3] = wd[1] * (3.0 * pi->K / wd[0] - wd[2] / 3.0);
    }
}

/* the force term p of bond b = (o -> q) of point o, as osb_force_point computes it */
static inline void osb_bond_term(const or_sys *sys, const or_state *st, int64_t o, int64_t b,
                                 const double *wd, double *p) {
    const double *x = st->pos;
    const or_params *po = P_of(sys, o);
    int32_t q = sys->nbr[b];
    double wvol = wd[4 * o], dil = wd[4 * o + 1], c1, c2;
    if (sys->multi) {
        const or_params *pq = P_of(sys, q);
        c1 = 15.0 * (po->G + pq->G) / (2 * wvol);
        c2 = dil * (3.0 * (po->K + pq->K) / (2 * wvol) - c1 / 3.0);
    } else {
        c1 = wd[4 * o + 2];
        c2 = wd[4 * o + 3];
    }
    double Lb = sys->L[b], l = st->bond_length[b];
    double d[3] = {x[3 * q] - x[3 * o], x[3 * q + 1] - x[3 * o + 1], x[3 * q + 2] - x[3 * o + 2]};
    double om = sys->omega[b] * (st->bond_active[b] ? 1.0 : 0.0);
    double s = om * SCF(sys, b) * (c2 * Lb + c1 * (l - Lb)) / l;
    for (int k = 0; k < 3; k++) p[k] = s * d[k];
}

/* the terms of point i's own bonds (zero when its weighted volume is zero) */
static void osb_terms_point(const or_sys *sys, const or_state *st, int64_t i, const double *wd,
                            double *pb) {
    for (int64_t b = sys->off[i]; b < sys->off[i + 1]; b++) {
        if (wd[4 * i] == 0.0) { pb[3 * b] = pb[3 * b + 1] = pb[3 * b + 2] = 0.0; continue; }
        osb_bond_term(sys, st, i, b, wd, pb + 3 * b);
    }
}

/* force row of point i in the serial loop's order from the stored bond terms */
static void gather_point(const or_sys *sys, or_state *st, int64_t i, const double *pb,
                         const unsigned char *live, const int64_t *rev) {
    double acc[3] = {0.0, 0.0, 0.0};
    const int64_t b0 = sys->off[i], b1 = sys->off[i + 1];
    for (int pass = 0; pass < 3; pass++)
        for (int64_t b = b0; b < b1; b++) {
            int32_t j = sys->nbr[b];
            if (pass == 1) {
                if (!live[i]) break;
                for (int k = 0; k < 3; k++) acc[k] += pb[3 * b + k] * sys->vol[j];
                continue;
            }
            if ((pass == 0) != (j < i) || !live[j]) continue;
            int64_t r = rev[b];
            if (r < 0) continue;
            for (int k = 0; k < 3; k++) acc[k] += -pb[3 * r + k] * sys->vol[j];
        }
    for (int k = 0; k < 3; k++) st->b_int[3 * i + k] = acc[k];
}

/* CMat point state (correspondence.jl:183-224, 288-298): F and P K^-1 into FP (18 per point),
 * alive[i] = 0 when the point's bonds are killed; defgrad, cauchy and the kill as
 * c_force_point */
/* per-point record of the serial-order gather: F (9), P K^-1 (9), ZEMWan's C_1 (9) */
#define C_FPS 27

static void c_state_point(const or_sys *sys, or_state *st, int64_t i, double *FP, unsigned char *alive) {
    const double *x = st->pos, *X = sys->X;
    const or_params *pi = P_of(sys, i);
    double K[9] = {0}, Ft[9] = {0};
    for (int64_t b = sys->off[i]; b < sys->off[i + 1]; b++) {
        int32_t j = sys->nbr[b];
        double D[3] = {X[3 * j] - X[3 * i], X[3 * j + 1] - X[3 * i + 1], X[3 * j + 2] - X[3 * i + 2]};
        double d[3] = {x[3 * j] - x[3 * i], x[3 * j + 1] - x[3 * i + 1], x[3 * j + 2] - x[3 * i + 2]};
        double om = sys->omega[b] * (st->bond_active[b] ? 1.0 : 0.0);
        double temp = om * sys->vol[j];
        for (int c = 0; c < 3; c++)
            for (int r = 0; r < 3; r++) {
                K[r + 3 * c] = K[r + 3 * c] + temp * (D[r] * D[c]);
                Ft[r + 3 * c] = Ft[r + 3 * c] + temp * (d[r] * D[c]);
            }
    }
    double Kinv[9], F[9];
    or_inv3(K, Kinv);
    matmul3(Ft, Kinv, F);
    memcpy(st->defgrad + 9 * i, F, sizeof(F));
    alive[i] = 1;
    if (st->damage[i] > sys->maxdmg || has_nan9(F)) {
        for (int64_t b = sys->off[i]; b < sys->off[i + 1]; b++) st->bond_active[b] = 0;
        st->n_active[i] = 0;
        alive[i] = 0;
        return;
    }
    double P[9], PKinv[9], PF[9];
    or_first_piola_kirchhoff(sys->cmodel, pi, F, P);
    matmul3(P, Kinv, PKinv);
    double J = or_det3(F), iJ = 1 / J, Ps[9];
    for (int k = 0; k < 9; k++) Ps[k] = iJ * P[k];
    matmulT3(Ps, F, PF);
    memcpy(st->cauchy + 9 * i, PF, sizeof(PF));
    memcpy(FP + C_FPS * i, F, sizeof(F));
    memcpy(FP + C_FPS * i + 9, PKinv, sizeof(PKinv));
    if (sys->zem == OR_ZEM_WAN) or_zem_wan_stiffness(pi, Kinv, FP + C_FPS * i + 18);
}

/* the force term t of bond b = (o -> q) of point o, as c_force_point computes it */
static inline void c_bond_term(const or_sys *sys, const or_state *st, int64_t o, int64_t b,
                               const double *FP, double *t) {
    const double *x = st->pos, *X = sys->X;
    const or_params *po = P_of(sys, o);
    int32_t q = sys->nbr[b];
    const double *F = FP + C_FPS * o, *PKinv = FP + C_FPS * o + 9, *C1 = FP + C_FPS * o + 18;
    double D[3] = {X[3 * q] - X[3 * o], X[3 * q + 1] - X[3 * o + 1], X[3 * q + 2] - X[3 * o + 2]};
    double d[3] = {x[3 * q] - x[3 * o], x[3 * q + 1] - x[3 * o + 1], x[3 * q + 2] - x[3 * o + 2]};
    double om = sys->omega[b] * (st->bond_active[b] ? 1.0 : 0.0);
    double FD[3], z[3], W[9], WD[3], tz[3];
    matvec3(F, D, FD);
    for (int k = 0; k < 3; k++) z[k] = d[k] - FD[k];
    zem_term(sys, po, C1, om, z, tz);
    for (int k = 0; k < 9; k++) W[k] = om * PKinv[k];
    matvec3(W, D, WD);
    for (int k = 0; k < 3; k++) t[k] = WD[k] + tz[k];
}

static void c_terms_point(const or_sys *sys, const or_state *st, int64_t i, const double *FP,
                          const unsigned char *alive, double *pb) {
    for (int64_t b = sys->off[i]; b < sys->off[i + 1]; b++) {
        if (!alive[i]) { pb[3 * b] = pb[3 * b + 1] = pb[3 * b + 2] = 0.0; continue; }
        c_bond_term(sys, st, i, b, FP, pb + 3 * b);
    }
}

/* reverse bond of every bond (-1 where the neighbour has no bond back), kept between calls
 * for the same bond arrays */
static int64_t *g_rev = NULL;
static const int32_t *g_rev_nbr = NULL;
static const int64_t *g_rev_off = NULL;
static int64_t g_rev_nb = -1;

static const int64_t *reverse_bonds(const or_sys *sys) {
    if (g_rev && g_rev_nbr == sys->nbr && g_rev_off == sys->off && g_rev_nb == sys->n_bonds)
        return g_rev;
    free(g_rev);
    g_rev = (int64_t *)malloc(sizeof(int64_t) * (size_t)(sys->n_bonds > 0 ? sys->n_bonds : 1));
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 1024)
    for (int64_t i = 0; i < sys->n; i++)
        for (int64_t b = sys->off[i]; b < sys->off[i + 1]; b++) g_rev[b] = reverse_bond(sys, sys->nbr[b], i);
    g_rev_nbr = sys->nbr;
    g_rev_off = sys->off;
    g_rev_nb = sys->n_bonds;
    return g_rev;
}

static void force_density_serial_order(const or_sys *sys, or_state *st) {
    int64_t n = sys->n;
    const int64_t *rev = reverse_bonds(sys);
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 1024)
    for (int64_t i = 0; i < n; i++) {
        st->n_active[i] = 0;
        failure_point(sys, st, i);
        damage_point(sys, st, i);
    }
    /* scratch kept between calls (a fresh allocation of this size per step costs more in page
     * faults than the step's arithmetic) */
    static double *pb = NULL;
    static size_t pb_cap = 0;
    size_t need = 3 * (size_t)(sys->n_bonds > 0 ? sys->n_bonds : 1);
    if (need > pb_cap) {
        free(pb);
        pb = (double *)malloc(sizeof(double) * need);
        pb_cap = need;
    }
    unsigned char *live = (unsigned char *)malloc((size_t)(n > 0 ? n : 1));
    if (sys->material == OR_OSB) {
        double *wd = (double *)malloc(sizeof(double) * 4 * (size_t)n);
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 1024)
        for (int64_t i = 0; i < n; i++) {
            osb_state_point(sys, st, i, wd + 4 * i);
            osb_coeffs_point(sys, i, wd + 4 * i);
            live[i] = wd[4 * i] != 0.0;
            osb_terms_point(sys, st, i, wd, pb);
        }
        free(wd);
    } else {
        double *FP = (double *)calloc((size_t)C_FPS * (size_t)(n > 0 ? n : 1), sizeof(double));
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 1024)
        for (int64_t i = 0; i < n; i++) {
            c_state_point(sys, st, i, FP, live);
            c_terms_point(sys, st, i, FP, live, pb);
        }
        free(FP);
    }
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 1024)
    for (int64_t i = 0; i < n; i++) gather_point(sys, st, i, pb, live, rev);
    free(live);
}

/* calc_force_density!: bond_system.jl:285-297 (one chunk), or the threads backend with
 * g_threads equal chunks for the scatter materials, or (or_set_serial_order) the serial
 * loop's order on g_threads threads. */
void or_force_density(const or_sys *sys, or_state *st, double t, double dt) {
    (void)t; (void)dt;
    int64_t n = sys->n;
    memset(st->b_int, 0, sizeof(double) * 3 * (size_t)n);
    if (g_serial_order && sys->material != OR_BB) {
        force_density_serial_order(sys, st);
        return;
    }
    if (sys->material == OR_BB || g_threads == 1 || n < 2 * g_threads) {
#pragma omp parallel for num_threads(sys->material == OR_BB ? g_threads : 1) schedule(static)
        for (int64_t i = 0; i < n; i++) {
            st->n_active[i] = 0;
            failure_point(sys, st, i);
            damage_point(sys, st, i);
            if (sys->material == OR_BB) bb_force_point(sys, st, i);
            else if (sys->material == OR_OSB) osb_force_point(sys, st, st->b_int, i);
            else c_force_point(sys, st, st->b_int, i);
        }
        return;
    }
    /* chunked scatter (threads backend): every chunk writes into its own buffer; the rows it
     * touched outside its own range are added to the owner afterwards */
    int nc = g_threads;
    double **buf = (double **)calloc((size_t)nc, sizeof(double *));
    int64_t *lo = (int64_t *)malloc(sizeof(int64_t) * nc), *hi = (int64_t *)malloc(sizeof(int64_t) * nc);
#pragma omp parallel num_threads(nc)
    {
#ifdef _OPENMP
        int c = omp_get_thread_num();
#else
        int c = 0;
#endif
        int64_t s = n * c / nc, e = n * (c + 1) / nc;
        /* touched range: own points and their neighbours */
        int64_t mn = s, mx = e - 1;
        for (int64_t i = s; i < e; i++)
            for (int64_t b = sys->off[i]; b < sys->off[i + 1]; b++) {
                if (sys->nbr[b] < mn) mn = sys->nbr[b];
                if (sys->nbr[b] > mx) mx = sys->nbr[b];
            }
        lo[c] = mn; hi[c] = mx;
        double *bb = (double *)calloc((size_t)(3 * (mx - mn + 1)), sizeof(double));
        buf[c] = bb;
        double *sink = bb - 3 * mn;
        for (int64_t i = s; i < e; i++) {
            st->n_active[i] = 0;
            failure_point(sys, st, i);
            damage_point(sys, st, i);
            if (sys->material == OR_OSB) osb_force_point(sys, st, sink, i);
            else c_force_point(sys, st, sink, i);
        }
#pragma omp barrier
        /* local rows first, then halo contributions of the other chunks in chunk order */
        for (int64_t i = s; i < e; i++)
            for (int k = 0; k < 3; k++) st->b_int[3 * i + k] = sink[3 * i + k];
        for (int c2 = 0; c2 < nc; c2++) {
            if (c2 == c) continue;
            int64_t a = lo[c2] > s ? lo[c2] : s, z = hi[c2] < e - 1 ? hi[c2] : e - 1;
            const double *o = buf[c2] - 3 * lo[c2];
            for (int64_t i = a; i <= z; i++)
                for (int k = 0; k < 3; k++) st->b_int[3 * i + k] += o[3 * i + k];
        }
#pragma omp barrier
        free(bb);
    }
    free(buf); free(lo); free(hi);
}

/* nans.jl:10-18 (b_int only) */
int or_contains_nan(const or_sys *sys, const or_state *st) {
    for (int64_t k = 0; k < 3 * sys->n; k++) if (isnan(st->b_int[k])) return 1;
    return 0;
}

/* calc_stable_timestep / calc_timestep_point: velocity_verlet.jl:136-163,
 * bond_system.jl:269-277 */
double or_stable_timestep(const or_sys *sys, double sf) {
    double dtmin = INFINITY;
    for (int64_t i = 0; i < sys->n; i++) {
        const or_params *p = P_of(sys, i);
        double dtsum = 0.0;
        for (int64_t b = sys->off[i]; b < sys->off[i + 1]; b++)
            dtsum += sys->vol[sys->nbr[b]] * p->bc / sys->L[b];
        double dti = sqrt(2 * p->rho / dtsum);
        if (dti < dtmin) dtmin = dti;
    }
    return dtmin * sf;
}

/* apply_boundary_conditions!: boundary_conditions.jl:37-51, 98-108, 198-226 */
static void apply_bcs(const or_sys *sys, or_state *st, const or_bc *bcs, int32_t n_bcs, int64_t step) {
    (void)sys;
    for (int32_t q = 0; q < n_bcs; q++) {
        const or_bc *bc = &bcs[q];
        double *field = bc->field == 0 ? st->vh : st->b_ext;
        for (int32_t k = 0; k < bc->n_pts; k++) {
            double v;
            if (bc->kind == 0) v = bc->values[step - bc->first_step];
            else if (bc->kind == 1) v = bc->values[(step - bc->first_step) * bc->n_pts + k];
            else v = bc->values[k];
            if (!isfinite(v)) continue;
            field[3 * (int64_t)bc->pts[k] + bc->dim] = v;
        }
    }
}

/* solve! / verlet_timestep!: velocity_verlet.jl:165-197, 239-295. Returns 0, or the step
 * number at which NaN values appeared in b_int (the state is left as the reference leaves
 * it when it throws NaNError: after the force evaluation of that step). */
int64_t or_run_vv(const or_sys *sys, or_state *st, const or_bc *bcs, int32_t n_bcs,
                  int64_t first_step, int64_t n_steps, double dt) {
    int64_t n = sys->n;
    double dth = 0.5 * dt;
    for (int64_t s = first_step; s < first_step + n_steps; s++) {
        double t = (double)s * dt;
#pragma omp parallel for num_threads(g_threads) schedule(static)
        for (int64_t k = 0; k < 3 * n; k++) st->vh[k] = st->v[k] + st->a[k] * dth;
        apply_bcs(sys, st, bcs, n_bcs, s);
#pragma omp parallel for num_threads(g_threads) schedule(static)
        for (int64_t k = 0; k < 3 * n; k++) {
            double du = st->vh[k] * dt;
            st->u[k] += du;
            st->pos[k] += du;
        }
        or_force_density(sys, st, t, dt);
        if (or_contains_nan(sys, st)) return s;
#pragma omp parallel for num_threads(g_threads) schedule(static)
        for (int64_t i = 0; i < n; i++) {
            double rho = P_of(sys, i)->rho;
            for (int k = 0; k < 3; k++) {
                int64_t d = 3 * i + k;
                st->a[d] = (st->b_int[d] + st->b_ext[d]) / rho;
                st->v[d] = st->vh[d] + st->a[d] * dth;
            }
        }
    }
    return 0;
}

/* ---------------------------------------------------------------------------------------
 * EnergySurfaceCorrection (src/discretization/bond_system_corrections.jl)
 * --------------------------------------------------------------------------------------- */

/* coordinate k of point j uniformly stretched by lam along dimension d (calc_mfactor! :101-104) */
static inline double stretched(const or_sys *sys, int64_t j, int k, int d, double lam) {
    return k == d ? lam * sys->X[3 * j + k] : sys->X[3 * j + k];
}

/* strain_energy_density_point! with scfactor = 1: BB (bond_based.jl:183-201) and OSB
 * (ordinary_state_based.jl:206-234, update_bond_lengths! :236-247) at the stretched positions */
static double esc_energy(const or_sys *sys, const or_state *st, int64_t i, int d, double lam) {
    const or_params *pi = P_of(sys, i);
    int64_t b0 = sys->off[i], b1 = sys->off[i + 1];
    double xi[3] = {stretched(sys, i, 0, d, lam), stretched(sys, i, 1, d, lam), stretched(sys, i, 2, d, lam)};
    if (sys->material == OR_BB) {
        double psi = 0.0;
        for (int64_t b = b0; b < b1; b++) {
            int32_t j = sys->nbr[b];
            double Lb = sys->L[b];
            double dx[3] = {stretched(sys, j, 0, d, lam) - xi[0], stretched(sys, j, 1, d, lam) - xi[1],
                            stretched(sys, j, 2, d, lam) - xi[2]};
            double l = sqrt(dot3(dx, dx));
            double eps = (l - Lb) / Lb;
            double om = bmul(st->bond_active[b], 1.0);
            double bc = (pi->bc + P_of(sys, j)->bc) / 2;
            psi += 0.25 * om * bc * eps * eps * Lb * sys->vol[j];
        }
        return psi;
    }
    const double *X = sys->X;
    double wvol = 0.0;
    for (int64_t b = b0; b < b1; b++) {
        int32_t j = sys->nbr[b];
        double D[3] = {X[3 * j] - X[3 * i], X[3 * j + 1] - X[3 * i + 1], X[3 * j + 2] - X[3 * i + 2]};
        double om = sys->omega[b] * (st->bond_active[b] ? 1.0 : 0.0);
        wvol += om * 1.0 * dot3(D, D) * sys->vol[j];
    }
    if (wvol == 0.0) return 0.0;  /* the density keeps its cleared value */
    double dil = 0.0, c1d = 3.0 / wvol;
    for (int64_t b = b0; b < b1; b++) {
        int32_t j = sys->nbr[b];
        double Lb = sys->L[b];
        double dx[3] = {stretched(sys, j, 0, d, lam) - xi[0], stretched(sys, j, 1, d, lam) - xi[1],
                        stretched(sys, j, 2, d, lam) - xi[2]};
        double l = sqrt(dot3(dx, dx));
        double om = sys->omega[b] * (st->bond_active[b] ? 1.0 : 0.0);
        dil += om * 1.0 * c1d * Lb * (l - Lb) * sys->vol[j];
    }
    double psivol = 0.5 * pi->K * (dil * dil);
    double psidev = 0.0;
    for (int64_t b = b0; b < b1; b++) {
        int32_t j = sys->nbr[b];
        double Lb = sys->L[b];
        double dx[3] = {stretched(sys, j, 0, d, lam) - xi[0], stretched(sys, j, 1, d, lam) - xi[1],
                        stretched(sys, j, 2, d, lam) - xi[2]};
        double l = sqrt(dot3(dx, dx));
        double e = l - Lb;
        double edev = e - 1.0 / 3.0 * dil * Lb;
        double om = sys->omega[b] * (st->bond_active[b] ? 1.0 : 0.0);
        double G = (pi->G + P_of(sys, j)->G) / 2;
        double cdev = 15.0 * G / (2 * wvol);
        psidev += cdev * om * 1.0 * edev * edev * sys->vol[j];
    }
    return psivol + psidev;
}

/* get_averaged_lame_parameters (:126-148): the point's (lambda, mu), or with several
 * parameter sets the mean over its active bonds of the bond-averaged pair */
void or_esc_lame(const or_sys *sys, const or_state *st, int64_t i, double *lame) {
    const or_params *pi = P_of(sys, i);
    lame[0] = pi->lambda;
    lame[1] = pi->mu;
    if (!sys->multi) return;
    double sl = 0.0, sm = 0.0;
    int64_t na = 0;
    for (int64_t b = sys->off[i]; b < sys->off[i + 1]; b++) {
        if (!st->bond_active[b]) continue;
        const or_params *pj = P_of(sys, sys->nbr[b]);
        sl += (pi->lambda + pj->lambda) / 2;
        sm += (pi->mu + pj->mu) / 2;
        na++;
    }
    lame[0] = sl / (double)na;
    lame[1] = sm / (double)na;
}

/* calc_mfactor! (:96-124) with stendens_uniext_small_strain (:150-152) */
void or_esc_mfactor(const or_sys *sys, const or_state *st, double *mfactor) {
    const double lam = 1.001;
    for (int d = 0; d < 3; d++) {
        for (int64_t i = 0; i < sys->n; i++) {
            double lame[2];
            or_esc_lame(sys, st, i, lame);
            double psi_theory = (0.5 * lame[0] + lame[1]) * ((lam - 1) * (lam - 1));
            mfactor[3 * i + d] = psi_theory / esc_energy(sys, st, i, d, lam);
        }
    }
}

/* calc_scfactor! (:156-204): the factor of bond i -> j from the mean mfactor of i and j in
 * the directions of the reference bond */
void or_esc_scfactor(const or_sys *sys, const double *mf, double *scfactor) {
    const double *X = sys->X;
    const double half_pi = 90 * M_PI / 180;
    for (int64_t i = 0; i < sys->n; i++) {
        for (int64_t b = sys->off[i]; b < sys->off[i + 1]; b++) {
            int32_t j = sys->nbr[b];
            double Lb = sys->L[b];
            double ax = fabs(X[3 * j] - X[3 * i]), ay = fabs(X[3 * j + 1] - X[3 * i + 1]),
                   az = fabs(X[3 * j + 2] - X[3 * i + 2]);
            double scx = (mf[3 * i] + mf[3 * j]) / 2;
            double scy = (mf[3 * i + 1] + mf[3 * j + 1]) / 2;
            double scz = (mf[3 * i + 2] + mf[3 * j + 2]) / 2;
            double scr, th, ph;
            if (az <= 1e-10) {
                if (ay <= 1e-10) th = 0.0;
                else if (ax <= 1e-10) th = half_pi;
                else th = atan(ay / ax);
                ph = half_pi;
            } else if (ax <= 1e-10 && ay <= 1e-10) {
                scfactor[b] = scz;
                continue;
            } else {
                th = atan(ay / ax);
                ph = acos(az / Lb);
            }
            double a = cos(th) * sin(ph), c = sin(th) * sin(ph), e = cos(ph);
            scr = sqrt(1 / ((a * a / (scx * scx) + c * c / (scy * scy)) + e * e / (scz * scz)));
            scfactor[b] = scr;
        }
    }
}
