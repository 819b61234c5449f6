/*
 * CPU oracle for the 2D GLM-MHD operator — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, FP64, single-threaded restatement of the reference CPU path
 * (MUSCL + HLL + Dedner GLM + Ohmic/Hall/ambipolar + SSP-RK2 + global CFL,
 * periodic/outflow ghost fill and the reflective solid-mask fill). It is the
 * checker the CUDA path is compared against; the product never links, loads
 * or calls it. Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it.
 *
 * State layout is the reference's StateField: 9 SoA planes, each
 * (ny + 2 ng) x (nx + 2 ng) doubles, row-major, index j * nx_tot + i
 * (include/state/state_field.hpp:9-73), planes in the order
 * rho, mx, my, mz, E, bx, by, bz, psi.
 *
 * Parity pin: tests/test_oracle_golden.py checks this code against the
 * reference's golden fixtures (tests/goldens/orszag_tang_32.golden and
 * ohmic_sine_bz_32.golden, via tests/golden/), and tests/test_oracle_vs_ref.py
 * against the reference CPU path compiled from its own headers into
 * oracle/_ref (oracle/ref_driver.cpp). The van Leer limiter has no reference
 * counterpart; its parity rests on this restatement alone.
 */
#ifndef MHD_ORACLE_H
#define MHD_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { MHDO_MINMOD = 0, MHDO_MC = 1, MHDO_VANLEER = 2 };
enum { MHDO_PERIODIC = 0, MHDO_REFLECTIVE = 1, MHDO_OUTFLOW = 2 };
enum { MHDO_OK = 0, MHDO_EINVAL = 1, MHDO_EMAXSTEPS = 2 };

typedef struct {
    int nx, ny, ng;
    double x_min, x_max, y_min, y_max;
} mhdo_grid;

typedef struct {
    double t_end, cfl, gamma, glm_alpha;
    int limiter;
    int ohmic, hall, ambipolar;
    double eta_ohm, eta_hall, eta_ambipolar;
    int max_steps;
    /* 1: run exactly max_steps steps with no t_end limit (t_end ignored). */
    int fixed_steps;
} mhdo_params;

typedef struct {
    double t;
    int steps;
    double c_h;
} mhdo_result;

typedef struct {
    double mass, energy;
    double div_b_max, div_b_l2;
    double rho_min, p_min;
    int finite;
} mhdo_diag;

/* Full solve, reference solve() semantics (include/mhd/time_integrator.hpp:62-106). */
int mhdo_solve(const mhdo_grid* g, const mhdo_params* p, int bc_x, int bc_y,
               const uint8_t* mask, int reflective_walls, double* U, mhdo_result* out);

/* One spatial-operator evaluation L(U) on the interior (ghost entries of rhs untouched). */
int mhdo_rhs(const mhdo_grid* g, const mhdo_params* p, const uint8_t* mask, double c_h,
             const double* U, double* rhs);

/* Ghost fill (boundary_conditions.hpp:90-103) and solid-wall fill (mask.hpp:85-149). */
int mhdo_apply_bc(const mhdo_grid* g, int bc_x, int bc_y, double* U);
int mhdo_wall_fill(const mhdo_grid* g, const uint8_t* mask, double gamma, double* U);

/* Global max signal speed and CFL dt (cfl.hpp:28-92). */
int mhdo_cfl(const mhdo_grid* g, const mhdo_params* p, const uint8_t* mask, const double* U,
             double* dt, double* c_h);

/* Slope limiter phi(a, b) (muscl_hll.hpp:33-57, plus van Leer). */
double mhdo_limiter(int kind, double a, double b);

/* Generalised Ohm's law E(J, B) of the non-ideal terms enabled in p (include/mhd/nonideal.hpp:
   63-102). */
void mhdo_nonideal_e(const double* J, const double* B, const mhdo_params* p, double* E);

/* Face flux from a 4-cell primitive stencil, x-frame order
   (rho, vn, vt, vz, p, bn, bt, bz, psi); out is the rotated-frame flux
   (rho, mn, mt, mz, E, bn, bt, bz, psi) (muscl_hll.hpp:126-209). */
void mhdo_face_flux(int limiter, const double* wmm, const double* wm, const double* w0,
                    const double* wp, double gamma, double c_h, double* out);

/* Interior diagnostics: mass/energy sums x dx dy, central-difference div B
   (inititial_condition.hpp:273-287) max and L2 (sqrt of mean square), min rho, min p. */
int mhdo_diagnostics(const mhdo_grid* g, double gamma, const double* U, mhdo_diag* out);

#ifdef __cplusplus
}
#endif

#endif
