/*
 * pd_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU FP64 restatement of Peridynamics.jl's explicit-dynamics hot path (bond search,
 * BB / OSB / correspondence force densities, critical-stretch failure, damage, Velocity
 * Verlet with boundary conditions, CFL time step, pre-cracks). It is the checker that the
 * CUDA library is compared against. Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference leg may load it; the product never calls it.
 *
 * The reference (pure Julia) cannot run in this container (no Julia toolchain). Parity of
 * this restatement is pinned against the reference's own known-answer tests, which the
 * files under tests/ reproduce (two-point BB/OSB force densities, the correspondence
 * regression values, the critical stretch of material!, the CFL time step, bond lists,
 * pre-crack damage).
 *
 * Compile with -ffp-contract=off: Julia does not contract a*b+c into an FMA, and the
 * restatement keeps Julia's operation order so that its rounding matches.
 */
#ifndef PD_ORACLE_H
#define PD_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* StandardPointParameters / CPointParameters minus the Hooke tensor
 * (src/core/parameters.jl:107-125, src/physics/correspondence.jl:148-161). */
typedef struct {
    double delta, rho, E, nu, G, K, lambda, mu, Gc, epsc, bc;
} or_params;

enum { OR_BB = 0, OR_OSB = 1, OR_CMAT = 2 };
enum { OR_SVK = 0, OR_NEOHOOKE = 1, OR_NHPENALTY = 2 };
enum { OR_KERNEL_CONST_ONE = 0, OR_KERNEL_LINEAR = 1, OR_KERNEL_CUBIC_BSPLINE = 2 };
enum { OR_ZEM_SILLING = 0, OR_ZEM_WAN = 1 };

typedef struct {
    int64_t n, n_bonds;
    const double *X;          /* 3n reference positions, xyz interleaved (Julia 3xN) */
    const double *vol;        /* n */
    const int64_t *off;       /* n+1 CSR offsets into the bond arrays */
    const int32_t *nbr;       /* B, 0-based neighbour index */
    const double *L;          /* B reference bond length */
    const uint8_t *fail_permit; /* B */
    const double *omega;      /* B kernel value per bond (OSB, CMat); may be NULL for BB */
    const int32_t *pid;       /* n parameter-set id per point */
    const or_params *params;  /* n_params */
    int32_t n_params;
    int32_t material;         /* OR_BB / OR_OSB / OR_CMAT */
    int32_t cmodel;           /* correspondence constitutive model */
    int32_t multi;            /* 1: ParameterHandler semantics (per-bond averaged parameters) */
    double zem_cs;            /* ZEMSilling Cs */
    double maxdmg;            /* CMaterial maxdmg */
    const double *scfactor;   /* B surface correction factor per bond; NULL: NoCorrection */
    int32_t zem;              /* CMat zero-energy mode stabilisation: OR_ZEM_SILLING, OR_ZEM_WAN */
} or_sys;

typedef struct {
    double *pos, *u, *v, *vh, *a, *b_int, *b_ext; /* 3n each */
    double *damage;           /* n */
    int64_t *n_active;        /* n */
    uint8_t *bond_active;     /* B */
    double *bond_length;      /* B (BB, OSB) */
    double *defgrad, *cauchy; /* 9n each (CMat), column-major 3x3 per point */
} or_state;

/* Boundary condition on one field/dim of a point list:
 * kind 0: one value per step (f(t) tabulated at t = n*dt), values[k]
 * kind 1: one value per point per step (f(p,t)), values[k*n_pts + q]
 * kind 2: one constant value per point (DataBC), values[q]
 * field 0: velocity_half, field 1: b_ext. A NaN / Inf value is skipped. */
typedef struct {
    int32_t field, dim, kind, n_pts;
    const int32_t *pts;
    const double *values;
    int64_t first_step;       /* step number of values[0] (kinds 0, 1) */
} or_bc;

int64_t or_find_bonds(int64_t n, const double *X, const double *delta, const uint8_t *fp_point,
                      const uint8_t *crack_a, const uint8_t *crack_b, int32_t n_cracks,
                      int64_t cap, int64_t *off, int32_t *nbr, double *L, uint8_t *fail_permit);
void or_kernels(const or_sys *sys, int32_t kernel, double *omega);
void or_init_state(const or_sys *sys, or_state *st);
void or_break_bonds(const or_sys *sys, or_state *st, const uint8_t *set_a, const uint8_t *set_b);
void or_calc_damage(const or_sys *sys, or_state *st);
void or_force_density(const or_sys *sys, or_state *st, double t, double dt);
int or_contains_nan(const or_sys *sys, const or_state *st);
double or_stable_timestep(const or_sys *sys, double safety_factor);
int64_t or_run_vv(const or_sys *sys, or_state *st, const or_bc *bcs, int32_t n_bcs,
                  int64_t first_step, int64_t n_steps, double dt);
void or_first_piola_kirchhoff(int32_t cmodel, const or_params *p, const double *F, double *P);
/* ZEMWan's stiffness C_1 = C : K^-1 of one point (zem_stabilization.jl:32-42) */
void or_zem_wan_stiffness(const or_params *p, const double *Kinv, double *C1);
void or_inv3(const double *A, double *Ainv);
double or_det3(const double *A);
int or_point_params(int32_t material, double delta, double rho, double E, double nu, double G,
                    double K, double lambda, double mu, double Gc, double epsc,
                    or_params *out, char *msg, int32_t msg_len);
void or_set_threads(int32_t n);
void or_set_serial_order(int32_t on);
/* EnergySurfaceCorrection (bond_system_corrections.jl): mfactor[3 i + d] of every point from the
 * current bond states (calc_mfactor!), and the per-bond factor from it (calc_scfactor!). */
void or_esc_mfactor(const or_sys *sys, const or_state *st, double *mfactor);
void or_esc_lame(const or_sys *sys, const or_state *st, int64_t i, double *lame);
void or_esc_scfactor(const or_sys *sys, const double *mfactor, double *scfactor);

#ifdef __cplusplus
}
#endif
#endif
