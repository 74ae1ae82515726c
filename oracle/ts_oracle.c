/* ORACLE (test infrastructure only): plain-C restatement of the treesap single-level
 * explicit integrator path, used as the checker of the B200 kernels. It is never linked
 * into the product.
 *
 * Every operation follows the reference's evaluation order, so that (compiled with
 * -ffp-contract=off) it reproduces the reference build (oracle/_ref/libtsref.so) bit for bit:
 *   stencil weights           util/stencil_impl.hpp:56-71 (first), :91-104 (second), cexprmath.hpp:32-105
 *   D1 / D2 / mixed D2        util/stencil_impl.hpp:192-223, :254-268, :269-286
 *   Kreiss-Oliger             util/stencil.hpp:77-104, rhs-decorators/KODecorator.hpp:58-70
 *   absorbing layer           rhs-decorators/ABLDecorator.hpp:85-132
 *   contract / symmetric idx  util/tensor_operations.hpp:45-61, tensor-alias/SymRank2Alias.hpp:41-62
 *   RK4 stage                 integrators/SingleLevelRK4Integrator.hpp:70-74, :115-158
 *   Euler                     integrators/SingleLevelEulerIntegrator.hpp:66-88
 *   ghost fill                SingleLevelIntegrator.hpp:153-163 + DirichletBC.hpp:43-65 / NoOpBC.hpp:41-46
 *                             (periodic images first, then the BC on cells outside the
 *                             domain grown in periodic directions only)
 *   initialisation            SingleLevelIntegrator.hpp:75-93 (cell centres lo + (i + 1/2) dx)
 * The model right-hand sides restate the built-in models (scalar wave with optional c(x)^2,
 * tensor wave) defined in treesap_b200/cpp/rhs/.
 */
#include "tsref.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef struct {
    int n[3], g, nc;
    long sx, sy, sz, sn; /* strides of the ghosted array [comp][z][y][x] */
    double dx[3];
} Grid;

static long at(const Grid* G, int i, int j, int k, int c) {
    return (long)(i + G->g) + (long)(j + G->g) * G->sy + (long)(k + G->g) * G->sz + (long)c * G->sn;
}

/* ------------------------------------------------------------------ weights */
static int64_t factorial(int n) {
    int64_t r = 1;
    for (int i = 2; i <= n; ++i) r *= i;
    return r;
}
static int64_t ipow(int64_t b, int e) {
    int64_t r = 1;
    while (e > 0) {
        if (e & 1) r *= b;
        b *= b;
        e >>= 1;
    }
    return r;
}
static int alt_sign(int k) { return (k & 1) ? -1 : 1; }
static int64_t binom(int n, int k) {
    if (k < 0 || k > n) return 0;
    if (k == 0 || k == n) return 1;
    if (k > n / 2) k = n - k;
    int64_t r = 1;
    for (int i = 1; i <= k; ++i) r = (r * (n - i + 1)) / i;
    return r;
}
static double harmonic2(int n) {
    double s = 0.0;
    for (int k = 1; k <= n; ++k) s += 1.0 / (double)ipow(k, 2);
    return s;
}
/* first-derivative weight for offset p > 0 (the p < 0 weight is its negative) */
static double w_first(int n, int p) {
    int64_t num = alt_sign(p + 1) * ipow(factorial(n), 2);
    int64_t den = p * factorial(n - p) * factorial(n + p);
    return (double)num / (double)den;
}
static double w_second(int n, int p) {
    if (p == 0) return -2.0 * harmonic2(n);
    int64_t num = 2 * alt_sign(p + 1) * ipow(factorial(n), 2);
    int64_t den = (int64_t)p * p * factorial(n - p) * factorial(n + p);
    return (double)num / (double)den;
}

/* ------------------------------------------------------------------ stencils */
static const int E[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};

static double d1(const Grid* G, const double* u, int c, int i, int j, int k, int d) {
    const double gf = 1.0 / G->dx[d];
    double st = 0.0;
    for (int s = 1; s <= G->g; ++s)
        st += w_first(G->g, s) * (u[at(G, i + s * E[d][0], j + s * E[d][1], k + s * E[d][2], c)] -
                                  u[at(G, i - s * E[d][0], j - s * E[d][1], k - s * E[d][2], c)]);
    return gf * st;
}

static double d2(const Grid* G, const double* u, int c, int i, int j, int k, int d0, int d1_) {
    if (d0 == d1_) {
        const double gf = 1.0 / (G->dx[d0] * G->dx[d0]);
        double st = w_second(G->g, 0) * u[at(G, i, j, k, c)];
        for (int s = 1; s <= G->g; ++s)
            st += w_second(G->g, s) * (u[at(G, i + s * E[d0][0], j + s * E[d0][1], k + s * E[d0][2], c)] +
                                       u[at(G, i - s * E[d0][0], j - s * E[d0][1], k - s * E[d0][2], c)]);
        return gf * st;
    }
    const double gf = 1.0 / G->dx[d0];
    double st = 0.0;
    for (int s = 1; s <= G->g; ++s)
        st += w_first(G->g, s) * (d1(G, u, c, i + s * E[d0][0], j + s * E[d0][1], k + s * E[d0][2], d1_) -
                                  d1(G, u, c, i - s * E[d0][0], j - s * E[d0][1], k - s * E[d0][2], d1_));
    return gf * st;
}

static double ko(const Grid* G, const double* u, int c, int i, int j, int k, int d) {
    const int r = G->g;
    const double norm = 1.0 / (double)ipow(2, 2 * r);
    const double gf = 1.0 / G->dx[d];
    double res = (double)(-binom(2 * r, r)) * u[at(G, i, j, k, c)];
    for (int s = 1; s <= r; ++s)
        res += (double)(-alt_sign(s) * binom(2 * r, r + s)) *
               (u[at(G, i + s * E[d][0], j + s * E[d][1], k + s * E[d][2], c)] +
                u[at(G, i - s * E[d][0], j - s * E[d][1], k - s * E[d][2], c)]);
    return res * norm * gf;
}

/* ------------------------------------------------------------------ models */
typedef struct {
    const tsref_desc* d;
    Grid G;
    int bulk_lo[3], bulk_hi[3];
    double inv_thickness;
} Model;

/* symmetric rank-2 alias: component of (a, b) relative to the alias base */
static int sym(int a, int b) {
    int row = a > b ? a : b, col = a > b ? b : a;
    return row * (row + 1) / 2 + col;
}
static const int SYM_ROW[6] = {0, 1, 1, 2, 2, 2};
static const int SYM_COL[6] = {0, 0, 1, 0, 1, 2};

static double rhs_undecorated(const Model* M, const double* u, int c, int i, int j, int k) {
    const Grid* G = &M->G;
    if (M->d->model == TSREF_MODEL_TENSOR_WAVE) {
        if (c < 6) return u[at(G, i, j, k, 6 + c)];
        const int q = c - 6, a0 = SYM_ROW[q], b0 = SYM_COL[q];
        double lap = 0.0;
        for (int a = 0; a < 3; ++a) lap += d2(G, u, sym(a0, b0), i, j, k, a, a);
        double div_i = 0.0, div_j = 0.0;
        for (int kk = 0; kk < 3; ++kk) div_i += d2(G, u, sym(kk, b0), i, j, k, a0, kk);
        for (int kk = 0; kk < 3; ++kk) div_j += d2(G, u, sym(kk, a0), i, j, k, b0, kk);
        double res = lap + 0.5 * (div_i + div_j);
        if (a0 == b0) {
            double lt = 0.0;
            for (int a = 0; a < 3; ++a) {
                double inner = 0.0;
                for (int kk = 0; kk < 3; ++kk) inner += d2(G, u, sym(kk, kk), i, j, k, a, a);
                lt += inner;
            }
            res -= (1.0 / 3.0) * lt;
        }
        return res;
    }
    if (c == 0) return u[at(G, i, j, k, 1)];
    double lap = 0.0;
    for (int a = 0; a < 3; ++a) lap += d2(G, u, 0, i, j, k, a, a);
    const double c2 = M->d->c2 ? M->d->c2[(long)i + (long)j * G->n[0] + (long)k * G->n[0] * G->n[1]] : 1.0;
    return c2 * lap;
}

static double sigma(const Model* M, int i, int j, int k) {
    const int idx[3] = {i, j, k};
    int inside = 1;
    for (int q = 0; q < 3; ++q)
        if (idx[q] < M->bulk_lo[q] || idx[q] > M->bulk_hi[q]) inside = 0;
    if (inside) return 0.0;
    int v[3];
    for (int q = 0; q < 3; ++q) {
        int cl = idx[q] < M->bulk_lo[q] ? M->bulk_lo[q] : (idx[q] > M->bulk_hi[q] ? M->bulk_hi[q] : idx[q]);
        v[q] = idx[q] - cl;
    }
    const double norm = sqrt((double)(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
    double s = M->inv_thickness * norm;
    s = s < 0.0 ? 0.0 : (s > 1.0 ? 1.0 : s);
    const double prof = (M->d->abl_profile == 1) ? s : s * s;
    return M->d->abl_max_strength * prof;
}

static double rhs(const Model* M, const double* u, int c, int i, int j, int k) {
    double r = rhs_undecorated(M, u, c, i, j, k);
    if (M->d->ko_strength > 0.0) {
        double kt = 0.0;
        kt += ko(&M->G, u, c, i, j, k, 0);
        kt += ko(&M->G, u, c, i, j, k, 1);
        kt += ko(&M->G, u, c, i, j, k, 2);
        r = r + M->d->ko_strength * kt;
    }
    if (M->d->abl_thickness > 0) r = r - sigma(M, i, j, k) * (u[at(&M->G, i, j, k, c)] - M->d->bc_values[c]);
    return r;
}

/* ------------------------------------------------------------------ ghost fill */
static void fill(const Model* M, double* u) {
    const Grid* G = &M->G;
    const tsref_desc* d = M->d;
    const int g = G->g;
    const int dirichlet = d->abl_thickness > 0 || d->bc == TSREF_BC_DIRICHLET;
    for (int k = -g; k < G->n[2] + g; ++k)
        for (int j = -g; j < G->n[1] + g; ++j)
            for (int i = -g; i < G->n[0] + g; ++i) {
                int p[3] = {i, j, k};
                int valid = 1;
                for (int q = 0; q < 3; ++q)
                    if (p[q] < 0 || p[q] >= G->n[q]) valid = 0;
                if (valid) continue;
                int s[3], inside = 1;
                for (int q = 0; q < 3; ++q) {
                    s[q] = p[q];
                    if (d->periodic[q]) s[q] = ((s[q] % G->n[q]) + G->n[q]) % G->n[q];
                    if (s[q] < 0 || s[q] >= G->n[q]) inside = 0;
                }
                if (inside) {
                    for (int c = 0; c < G->nc; ++c) u[at(G, i, j, k, c)] = u[at(G, s[0], s[1], s[2], c)];
                } else if (dirichlet) {
                    for (int c = 0; c < G->nc; ++c) u[at(G, i, j, k, c)] = d->bc_values[c];
                }
            }
}

/* ------------------------------------------------------------------ driver */
static double now_seconds(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int tso_run(const tsref_desc* d, int init_kind, int nitems, const double* items, const double* state_in, int nsteps,
            double* state_out, double* seconds, double* time_out) {
    if (!d || !state_out || nsteps < 0 || d->ngrow < 1 || d->ngrow > 4) return 1;
    if (init_kind == TSREF_INIT_STATE && !state_in) return 1;
    Model M;
    memset(&M, 0, sizeof M);
    M.d = d;
    Grid* G = &M.G;
    G->g = d->ngrow;
    G->nc = (d->model == TSREF_MODEL_TENSOR_WAVE) ? 12 : 2;
    for (int q = 0; q < 3; ++q) {
        G->n[q] = d->n[q];
        if (G->n[q] < G->g) return 1;
        G->dx[q] = (d->prob_hi[q] - d->prob_lo[q]) / (double)d->n[q];
        M.bulk_lo[q] = d->abl_thickness;
        M.bulk_hi[q] = d->n[q] - 1 - d->abl_thickness;
    }
    if (d->abl_thickness > 0) M.inv_thickness = 1.0 / (double)d->abl_thickness;
    G->sx = 1;
    G->sy = G->n[0] + 2 * G->g;
    G->sz = G->sy * (G->n[1] + 2 * G->g);
    G->sn = G->sz * (G->n[2] + 2 * G->g);
    const long total = G->sn * G->nc;
    const long ncell = (long)G->n[0] * G->n[1] * G->n[2];

    double* u = calloc((size_t)total, sizeof(double));
    double* acc = calloc((size_t)total, sizeof(double));
    double* arg = calloc((size_t)total, sizeof(double));
    double* argn = calloc((size_t)total, sizeof(double));
    if (!u || !acc || !arg || !argn) {
        free(u), free(acc), free(arg), free(argn);
        return 3;
    }

    /* initialise at cell centres */
    for (int k = 0; k < G->n[2]; ++k)
        for (int j = 0; j < G->n[1]; ++j)
            for (int i = 0; i < G->n[0]; ++i) {
                const long q = (long)i + (long)j * G->n[0] + (long)k * G->n[0] * G->n[1];
                const double x = d->prob_lo[0] + (i + 0.5) * G->dx[0];
                const double y = d->prob_lo[1] + (j + 0.5) * G->dx[1];
                const double z = d->prob_lo[2] + (k + 0.5) * G->dx[2];
                for (int c = 0; c < G->nc; ++c) {
                    double v = 0.0;
                    if (init_kind == TSREF_INIT_STATE) {
                        v = state_in[c * ncell + q];
                    } else if (init_kind == TSREF_INIT_GAUSSIAN) {
                        for (int p = 0; p < nitems; ++p) {
                            const double* it = items + 6 * p;
                            if ((int)it[0] != c) continue;
                            const double ex = x - it[3], ey = y - it[4], ez = z - it[5];
                            v += it[1] * exp(-(ex * ex + ey * ey + ez * ez) / (it[2] * it[2]));
                        }
                    } else {
                        const double two_pi = 6.283185307179586476925286766559;
                        for (int m = 0; m < nitems; ++m) {
                            const double* it = items + 6 * m;
                            if ((int)it[0] != c) continue;
                            v += it[1] * cos(two_pi * (it[2] * x + it[3] * y + it[4] * z) + it[5]);
                        }
                    }
                    u[at(G, i, j, k, c)] = v;
                }
            }

    static const double a_frac[4] = {0.0, 0.5, 0.5, 1.0};
    static const double b_frac[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
    double time = 0.0;
    const double dt = d->dt;
    const double t0 = now_seconds();
    for (int step = 0; step < nsteps; ++step) {
        fill(&M, u);
        if (d->integrator == TSREF_EULER) {
            for (int k = 0; k < G->n[2]; ++k)
                for (int j = 0; j < G->n[1]; ++j)
                    for (int i = 0; i < G->n[0]; ++i)
                        for (int c = 0; c < G->nc; ++c)
                            acc[at(G, i, j, k, c)] = u[at(G, i, j, k, c)] + dt * rhs(&M, u, c, i, j, k);
        } else {
            for (int s = 0; s < 4; ++s) {
                const double a_next = dt * a_frac[(s + 1) % 4];
                const double b = dt * b_frac[s];
                if (s > 0) {
                    double* t = arg;
                    arg = argn;
                    argn = t;
                    fill(&M, arg);
                }
                const double* src = (s == 0) ? u : arg;
                for (int k = 0; k < G->n[2]; ++k)
                    for (int j = 0; j < G->n[1]; ++j)
                        for (int i = 0; i < G->n[0]; ++i)
                            for (int c = 0; c < G->nc; ++c) {
                                const long o = at(G, i, j, k, c);
                                const double stage = rhs(&M, src, c, i, j, k);
                                if (s == 0)
                                    acc[o] = u[o] + b * stage;
                                else
                                    acc[o] += b * stage;
                                if (s < 3) argn[o] = u[o] + a_next * stage;
                            }
            }
        }
        double* t = u;
        u = acc;
        acc = t;
        time += dt;
    }
    const double t1 = now_seconds();

    for (int c = 0; c < G->nc; ++c)
        for (int k = 0; k < G->n[2]; ++k)
            for (int j = 0; j < G->n[1]; ++j)
                for (int i = 0; i < G->n[0]; ++i)
                    state_out[c * ncell + (long)i + (long)j * G->n[0] + (long)k * G->n[0] * G->n[1]] =
                        u[at(G, i, j, k, c)];
    if (seconds) *seconds = t1 - t0;
    if (time_out) *time_out = time;
    free(u), free(acc), free(arg), free(argn);
    return 0;
}

int tso_threads(void) { return 1; }
