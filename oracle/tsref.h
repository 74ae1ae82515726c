/* ORACLE interface (test infrastructure only; never linked into the product).
 *
 * Two CPU implementations of the single-level explicit integrator path export the same
 * entry point `*_run` with this descriptor:
 *   oracle/_ref/libtsref.so      the reference's own headers (src/treesap/**) compiled unchanged
 *                                against the host AMReX-API shim in oracle/amrex_host/;
 *   oracle/_build/libtsoracle.so a plain-C restatement of the same algorithm (ts_oracle.c).
 *
 * State arrays hold the valid cells only, component-major: [comp][z][y][x], x fastest.
 */
#ifndef TSREF_H
#define TSREF_H

#ifdef __cplusplus
extern "C" {
#endif

enum { TSREF_MODEL_WAVE = 0, TSREF_MODEL_TENSOR_WAVE = 1 };
enum { TSREF_INIT_STATE = 0, TSREF_INIT_GAUSSIAN = 1, TSREF_INIT_FOURIER = 2 };
enum { TSREF_EULER = 0, TSREF_RK4 = 1 };
enum { TSREF_BC_NOOP = 0, TSREF_BC_DIRICHLET = 1 };

typedef struct tsref_desc {
    int n[3];               /* valid cells per direction; index range 0..n-1 */
    double prob_lo[3];      /* physical domain */
    double prob_hi[3];
    int periodic[3];        /* 1: periodic in that direction */
    int ngrow;              /* stencil half-width = ghost width, 1..4 */
    int model;              /* TSREF_MODEL_* */
    double ko_strength;     /* > 0: KODecorator{rhs, ko_strength} with order = ngrow */
    int abl_thickness;      /* > 0: ABLPDEModel (absorbing layer, Dirichlet(target) ghosts) */
    double abl_max_strength;
    int abl_profile;        /* 1: s, 2: s^2 */
    int bc;                 /* TSREF_BC_* (ignored when the absorbing layer is on) */
    double bc_values[12];   /* Dirichlet values; absorbing-layer targets */
    double dt;
    int integrator;         /* TSREF_EULER / TSREF_RK4 */
    int block[3];           /* block_size of SingleLevelIntegrator; <= 0: whole domain */
    const double* c2;       /* scalar wave only: NULL = unit speed, else speed^2 per valid cell */
} tsref_desc;

/* Initialise (init_kind: TSREF_INIT_STATE copies state_in; GAUSSIAN: nitems pulses of
 * 6 doubles {comp, A, w, cx, cy, cz}; FOURIER: nitems modes of 6 doubles
 * {comp, A, kx, ky, kz, phase}), advance nsteps steps, write the final valid state to
 * state_out. *seconds receives the host wall time of the step loop, *time_out the
 * integrator's simulation time. Returns 0 on success, nonzero on an invalid descriptor. */
int tsref_run(const tsref_desc* d, int init_kind, int nitems, const double* items, const double* state_in,
              int nsteps, double* state_out, double* seconds, double* time_out);
int tso_run(const tsref_desc* d, int init_kind, int nitems, const double* items, const double* state_in,
            int nsteps, double* state_out, double* seconds, double* time_out);

/* Number of host threads the implementation uses. */
int tsref_threads(void);
int tso_threads(void);

#ifdef __cplusplus
}
#endif
#endif
