/*
 * CPU oracle for the 2D GLM-MHD operator — TEST INFRASTRUCTURE ONLY (see mhd_oracle.h).
 *
 * Plain C99, FP64. Every function cites the reference file:line it restates (paths relative to
 * the reference project root). Built with OpenMP, the loops over cells, rows and faces run on all
 * host threads: every value they write depends only on inputs of the same pass, so the results do
 * not depend on the thread count; the CFL maximum is combined per row, and the diagnostics sums
 * run in one thread in row order. Face fluxes are kept in full-grid arrays
 * instead of the reference's three rolling rows (include/mhd/rhs.hpp:186-239); each face is
 * still evaluated once from the same four cells, so the arithmetic is the same.
 */
#include "mhd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NF 9
enum { C_RHO = 0, C_MX, C_MY, C_MZ, C_E, C_BX, C_BY, C_BZ, C_PSI };

typedef struct {
    double rho, vn, vt, vz, p, bn, bt, bz, psi;
} primn;

typedef struct {
    double rho, mn, mt, mz, e, bn, bt, bz, psi;
} fluxn;

/* mhd::simd scalar helpers (include/mhd/simd.hpp:40-59). */
static double vmin(double a, double b) { return (b < a) ? b : a; }
static double vmax(double a, double b) { return (a < b) ? b : a; }

/* ---------------------------------------------------------------- limiters */

/* include/mhd/kernels/muscl_hll.hpp:33-38 */
static double minmod(double a, double b)
{
    return (a * b <= 0.0) ? 0.0 : ((fabs(a) < fabs(b)) ? a : b);
}

/* include/mhd/kernels/muscl_hll.hpp:41-47 */
static double mc_limiter(double a, double b)
{
    return minmod(0.5 * (a + b), minmod(2.0 * a, 2.0 * b));
}

/* van Leer (1974) harmonic limiter: 2ab/(a+b) when a, b share a sign, else 0.
   No reference counterpart (the reference offers only Minmod and MC,
   include/mhd/mhd_types.hpp:44). */
static double vanleer_limiter(double a, double b)
{
    return (a * b <= 0.0) ? 0.0 : (2.0 * a * b) / (a + b);
}

double mhdo_limiter(int kind, double a, double b)
{
    switch (kind) {
    case MHDO_MINMOD:
        return minmod(a, b);
    case MHDO_MC:
        return mc_limiter(a, b);
    default:
        return vanleer_limiter(a, b);
    }
}

/* include/mhd/kernels/muscl_hll.hpp:59-68 */
static void reconstruct(int lim, double wmm, double wm, double w0, double wp, double* left,
                        double* right)
{
    const double dm = mhdo_limiter(lim, wm - wmm, w0 - wm);
    const double d0 = mhdo_limiter(lim, w0 - wm, wp - w0);
    *left = wm + 0.5 * dm;
    *right = w0 - 0.5 * d0;
}

/* ---------------------------------------------------------------- point physics */

/* include/mhd/kernels/muscl_hll.hpp:70-87 */
static double fast_speed_n(const primn* W, double gamma)
{
    const double inv_rho = 1.0 / W->rho;
    const double cs2 = gamma * W->p * inv_rho;
    const double bn2 = W->bn * W->bn;
    const double b2 = bn2 + W->bt * W->bt + W->bz * W->bz;
    const double va2 = b2 * inv_rho;
    const double van2 = bn2 * inv_rho;
    const double sum = cs2 + va2;
    const double disc = vmax(sum * sum - 4.0 * cs2 * van2, 0.0);
    const double cf2 = 0.5 * (sum + sqrt(disc));
    return sqrt(vmax(cf2, 0.0));
}

/* include/mhd/kernels/muscl_hll.hpp:89-124 */
static void conserved_and_flux(const primn* W, double inv_gm1, double ch2, fluxn* U, fluxn* F)
{
    const double mn = W->rho * W->vn;
    const double mt = W->rho * W->vt;
    const double mz = W->rho * W->vz;
    const double v2 = W->vn * W->vn + W->vt * W->vt + W->vz * W->vz;
    const double b2 = W->bn * W->bn + W->bt * W->bt + W->bz * W->bz;
    const double pmag = 0.5 * b2;
    const double energy = W->p * inv_gm1 + 0.5 * W->rho * v2 + pmag;
    const double pstar = W->p + pmag;
    const double vb = W->vn * W->bn + W->vt * W->bt + W->vz * W->bz;

    U->rho = W->rho;
    U->mn = mn;
    U->mt = mt;
    U->mz = mz;
    U->e = energy;
    U->bn = W->bn;
    U->bt = W->bt;
    U->bz = W->bz;
    U->psi = W->psi;

    F->rho = mn;
    F->mn = mn * W->vn + pstar - W->bn * W->bn;
    F->mt = mn * W->vt - W->bn * W->bt;
    F->mz = mn * W->vz - W->bn * W->bz;
    F->e = (energy + pstar) * W->vn - W->bn * vb + W->psi * W->bn;
    F->bn = W->psi;
    F->bt = W->vn * W->bt - W->vt * W->bn;
    F->bz = W->vn * W->bz - W->vz * W->bn;
    F->psi = ch2 * W->bn;
}

static double hll_combine(double fl, double fr, double ul, double ur, double sL, double sR,
                          double sLsR, double inv_denom, int use_left, int use_right,
                          int degenerate)
{
    /* include/mhd/kernels/muscl_hll.hpp:192-196 */
    const double hll = (sR * fl - sL * fr + sLsR * (ur - ul)) * inv_denom;
    const double mid = degenerate ? 0.5 * (fl + fr) : hll;
    return use_left ? fl : (use_right ? fr : mid);
}

/* include/mhd/kernels/muscl_hll.hpp:126-209 */
static fluxn muscl_hll_face(int lim, const primn* Wmm, const primn* Wm, const primn* W0,
                            const primn* Wp, double gamma, double inv_gm1, double c_h)
{
    primn WL, WR;
    reconstruct(lim, Wmm->rho, Wm->rho, W0->rho, Wp->rho, &WL.rho, &WR.rho);
    reconstruct(lim, Wmm->vn, Wm->vn, W0->vn, Wp->vn, &WL.vn, &WR.vn);
    reconstruct(lim, Wmm->vt, Wm->vt, W0->vt, Wp->vt, &WL.vt, &WR.vt);
    reconstruct(lim, Wmm->vz, Wm->vz, W0->vz, Wp->vz, &WL.vz, &WR.vz);
    reconstruct(lim, Wmm->p, Wm->p, W0->p, Wp->p, &WL.p, &WR.p);
    reconstruct(lim, Wmm->bn, Wm->bn, W0->bn, Wp->bn, &WL.bn, &WR.bn);
    reconstruct(lim, Wmm->bt, Wm->bt, W0->bt, Wp->bt, &WL.bt, &WR.bt);
    reconstruct(lim, Wmm->bz, Wm->bz, W0->bz, Wp->bz, &WL.bz, &WR.bz);
    reconstruct(lim, Wmm->psi, Wm->psi, W0->psi, Wp->psi, &WL.psi, &WR.psi);

    /* Positivity and finiteness of both face states, else first order on both sides
       (muscl_hll.hpp:145-168). */
    const int ok = (WL.rho > 0.0) && (WL.p > 0.0) && (WL.rho < HUGE_VAL) && (WL.p < HUGE_VAL) &&
                   (WR.rho > 0.0) && (WR.p > 0.0) && (WR.rho < HUGE_VAL) && (WR.p < HUGE_VAL);
    if (!ok) {
        WL = *Wm;
        WR = *W0;
    }

    const double cfL = fast_speed_n(&WL, gamma);
    const double cfR = fast_speed_n(&WR, gamma);
    const double sL = vmin(vmin(WL.vn - cfL, WR.vn - cfR), -c_h);
    const double sR = vmax(vmax(WL.vn + cfL, WR.vn + cfR), c_h);

    const double ch2 = c_h * c_h;
    fluxn UL, UR, FL, FR;
    conserved_and_flux(&WL, inv_gm1, ch2, &UL, &FL);
    conserved_and_flux(&WR, inv_gm1, ch2, &UR, &FR);

    const double denom = sR - sL;
    const double inv_denom = 1.0 / denom;
    const double sLsR = sL * sR;
    const int use_left = sL >= 0.0;
    const int use_right = sR <= 0.0;
    const int degenerate = fabs(denom) < 1.0e-14;

    fluxn F;
#define COMB(f) F.f = hll_combine(FL.f, FR.f, UL.f, UR.f, sL, sR, sLsR, inv_denom, use_left, use_right, degenerate)
    COMB(rho);
    COMB(mn);
    COMB(mt);
    COMB(mz);
    COMB(e);
    COMB(bn);
    COMB(bt);
    COMB(bz);
    COMB(psi);
#undef COMB
    return F;
}

void mhdo_face_flux(int limiter, const double* wmm, const double* wm, const double* w0,
                    const double* wp, double gamma, double c_h, double* out)
{
    primn a, b, c, d;
    memcpy(&a, wmm, sizeof a);
    memcpy(&b, wm, sizeof b);
    memcpy(&c, w0, sizeof c);
    memcpy(&d, wp, sizeof d);
    const fluxn F = muscl_hll_face(limiter, &a, &b, &c, &d, gamma, 1.0 / (gamma - 1.0), c_h);
    memcpy(out, &F, sizeof F);
}

/* include/mhd/kernels/muscl_hll.hpp:211-239 */
static double cell_max_signal_speed(double rho, double mx, double my, double mz, double energy,
                                    double bx, double by, double bz, double gamma)
{
    const double inv_rho = 1.0 / rho;
    primn W;
    W.rho = rho;
    W.vn = mx * inv_rho;
    W.vt = my * inv_rho;
    W.vz = mz * inv_rho;
    const double ekin = 0.5 * (mx * mx + my * my + mz * mz) * inv_rho;
    const double emag = 0.5 * (bx * bx + by * by + bz * bz);
    W.p = (gamma - 1.0) * (energy - ekin - emag);
    W.bn = bx;
    W.bt = by;
    W.bz = bz;
    W.psi = 0.0;
    const double sx = fabs(W.vn) + fast_speed_n(&W, gamma);
    primn Wy = W;
    Wy.vn = W.vt;
    Wy.vt = W.vn;
    Wy.bn = by;
    Wy.bt = bx;
    const double sy = fabs(Wy.vn) + fast_speed_n(&Wy, gamma);
    return vmax(sx, sy);
}

/* ---------------------------------------------------------------- grid helpers */

typedef struct {
    int nx, ny, ng, nxt, nyt;
    size_t n;
    double dx, dy;
} geom;

static int make_geom(const mhdo_grid* g, geom* G)
{
    if (g == NULL || g->nx < 1 || g->ny < 1 || g->ng < 2) {
        return MHDO_EINVAL;
    }
    G->nx = g->nx;
    G->ny = g->ny;
    G->ng = g->ng;
    G->nxt = g->nx + 2 * g->ng;
    G->nyt = g->ny + 2 * g->ng;
    G->n = (size_t)G->nxt * (size_t)G->nyt;
    /* include/grid/grid.hpp:168-174 */
    G->dx = (g->x_max - g->x_min) / (double)g->nx;
    G->dy = (g->y_max - g->y_min) / (double)g->ny;
    return MHDO_OK;
}

static size_t at(const geom* G, int i, int j) { return (size_t)j * (size_t)G->nxt + (size_t)i; }

static void copy_cell(const geom* G, double* U, int id, int jd, int is, int js)
{
    const size_t d = at(G, id, jd), s = at(G, is, js);
    for (int c = 0; c < NF; ++c) {
        U[(size_t)c * G->n + d] = U[(size_t)c * G->n + s];
    }
}

/* include/boundary_conditions/boundary_conditions.hpp:26-30 */
static int periodic_source(int g, int n, int ng, int low)
{
    const int offset = low ? (g - ng) : g;
    return ng + ((offset % n) + n) % n;
}

/* include/boundary_conditions/boundary_conditions.hpp:32-103: x ghosts over every row first,
   then y ghosts over the full x range (corners come from the already filled x ghosts). */
int mhdo_apply_bc(const mhdo_grid* g, int bc_x, int bc_y, double* U)
{
    geom G;
    if (make_geom(g, &G) != MHDO_OK || bc_x == MHDO_REFLECTIVE || bc_y == MHDO_REFLECTIVE) {
        return MHDO_EINVAL;
    }
    for (int j = 0; j < G.nyt; ++j) {
        for (int gg = 0; gg < G.ng; ++gg) {
            const int il = gg, ir = G.ng + G.nx + gg;
            if (bc_x == MHDO_PERIODIC) {
                copy_cell(&G, U, il, j, periodic_source(gg, G.nx, G.ng, 1), j);
                copy_cell(&G, U, ir, j, periodic_source(gg, G.nx, G.ng, 0), j);
            } else {
                copy_cell(&G, U, il, j, G.ng, j);
                copy_cell(&G, U, ir, j, G.ng + G.nx - 1, j);
            }
        }
    }
    for (int i = 0; i < G.nxt; ++i) {
        for (int gg = 0; gg < G.ng; ++gg) {
            const int jb = gg, jt = G.ng + G.ny + gg;
            if (bc_y == MHDO_PERIODIC) {
                copy_cell(&G, U, i, jb, i, periodic_source(gg, G.ny, G.ng, 1));
                copy_cell(&G, U, i, jt, i, periodic_source(gg, G.ny, G.ng, 0));
            } else {
                copy_cell(&G, U, i, jb, i, G.ng);
                copy_cell(&G, U, i, jt, i, G.ng + G.ny - 1);
            }
        }
    }
    return MHDO_OK;
}

static int mask_active(const geom* G, const uint8_t* mask)
{
    if (mask == NULL) {
        return 0;
    }
    const size_t m = (size_t)G->nx * (size_t)G->ny;
    for (size_t k = 0; k < m; ++k) {
        if (mask[k] == 0) {
            return 1;
        }
    }
    return 0;
}

/* include/mask.hpp:55-64 (global indices; ghosts count as fluid). */
static int is_fluid_global(const geom* G, const uint8_t* mask, int i, int j)
{
    const int ii = i - G->ng, jj = j - G->ng;
    if (ii < 0 || jj < 0 || ii >= G->nx || jj >= G->ny) {
        return 1;
    }
    return mask[(size_t)jj * (size_t)G->nx + (size_t)ii] != 0;
}

/* include/mhd/mhd_physics.hpp:23-57 (to_primitive / to_conservative, division form). */
static void set_conservative_from_primitive(const geom* G, double* U, size_t d, double rho,
                                            double vx, double vy, double vz, double p, double bx,
                                            double by, double bz, double psi, double gamma)
{
    const double e_kin = 0.5 * rho * (vx * vx + vy * vy + vz * vz);
    const double e_mag = 0.5 * (bx * bx + by * by + bz * bz);
    U[0 * G->n + d] = rho;
    U[1 * G->n + d] = rho * vx;
    U[2 * G->n + d] = rho * vy;
    U[3 * G->n + d] = rho * vz;
    U[4 * G->n + d] = p / (gamma - 1.0) + e_kin + e_mag;
    U[5 * G->n + d] = bx;
    U[6 * G->n + d] = by;
    U[7 * G->n + d] = bz;
    U[8 * G->n + d] = psi;
}

/* include/mhd/mask.hpp:85-149: each solid interior cell copies its first fluid interior
   neighbour in the order +x, -x, +y, -y, with the normal velocity negated and rho, p floored
   at 1e-12; with no fluid neighbour it becomes rho = p = 1 at rest with zero fields. */
int mhdo_wall_fill(const mhdo_grid* g, const uint8_t* mask, double gamma, double* U)
{
    geom G;
    if (make_geom(g, &G) != MHDO_OK) {
        return MHDO_EINVAL;
    }
    if (!mask_active(&G, mask)) {
        return MHDO_OK;
    }
    const int ib = G.ng, ie = G.ng + G.nx, jb = G.ng, je = G.ng + G.ny;
    for (int j = jb; j < je; ++j) {
        for (int i = ib; i < ie; ++i) {
            if (is_fluid_global(&G, mask, i, j)) {
                continue;
            }
            const int cand[4][3] = {{i + 1, j, 0}, {i - 1, j, 0}, {i, j + 1, 1}, {i, j - 1, 1}};
            int filled = 0;
            for (int k = 0; k < 4; ++k) {
                const int ni = cand[k][0], nj = cand[k][1], axis = cand[k][2];
                if (ni < ib || ni >= ie || nj < jb || nj >= je) {
                    continue;
                }
                if (!is_fluid_global(&G, mask, ni, nj)) {
                    continue;
                }
                const size_t s = at(&G, ni, nj);
                const double rho = U[0 * G.n + s];
                const double mx = U[1 * G.n + s], my = U[2 * G.n + s], mz = U[3 * G.n + s];
                const double E = U[4 * G.n + s];
                const double bx = U[5 * G.n + s], by = U[6 * G.n + s], bz = U[7 * G.n + s];
                const double psi = U[8 * G.n + s];
                double vx = mx / rho, vy = my / rho;
                const double vz = mz / rho;
                const double e_kin = 0.5 * (mx * mx + my * my + mz * mz) / rho;
                const double e_mag = 0.5 * (bx * bx + by * by + bz * bz);
                double p = (gamma - 1.0) * (E - e_kin - e_mag);
                double r = rho;
                if (axis == 0) {
                    vx = -vx;
                } else {
                    vy = -vy;
                }
                if (r < 1e-12) {
                    r = 1e-12;
                }
                if (p < 1e-12) {
                    p = 1e-12;
                }
                set_conservative_from_primitive(&G, U, at(&G, i, j), r, vx, vy, vz, p, bx, by, bz,
                                                psi, gamma);
                filled = 1;
                break;
            }
            if (!filled) {
                set_conservative_from_primitive(&G, U, at(&G, i, j), 1.0, 0.0, 0.0, 0.0, 1.0, 0.0,
                                                0.0, 0.0, 0.0, gamma);
            }
        }
    }
    return MHDO_OK;
}

/* ---------------------------------------------------------------- CFL */

static double max_diffusivity(const mhdo_params* p)
{
    /* include/physics_config/mhd_config.hpp:97-110 */
    double eta = 0.0;
    if (p->ohmic) {
        eta = vmax(eta, fabs(p->eta_ohm));
    }
    if (p->hall) {
        eta = vmax(eta, fabs(p->eta_hall));
    }
    if (p->ambipolar) {
        eta = vmax(eta, fabs(p->eta_ambipolar));
    }
    return eta;
}

static int nonideal_any(const mhdo_params* p)
{
    /* include/physics_config/mhd_config.hpp:90-94 */
    return (p->ohmic && p->eta_ohm != 0.0) || (p->hall && p->eta_hall != 0.0) ||
           (p->ambipolar && p->eta_ambipolar != 0.0);
}

/* include/mhd/cfl.hpp:28-92 */
static void cfl_dt(const geom* G, const mhdo_params* p, const uint8_t* mask, const double* U,
                   double* dt_out, double* ch_out)
{
    const double inv_dx = 1.0 / G->dx;
    const double inv_dy = 1.0 / G->dy;
    /* per-row maxima (any thread may take any row), then the maximum over the rows in order */
    double* row_max = (double*)malloc((size_t)G->ny * sizeof(double));
    if (row_max == NULL) {
        *dt_out = NAN; /* the solve loop rejects a dt that is not positive */
        *ch_out = NAN;
        return;
    }
    #pragma omp parallel for schedule(static)
    for (int j = G->ng; j < G->ng + G->ny; ++j) {
        double m = 0.0;
        for (int i = G->ng; i < G->ng + G->nx; ++i) {
            if (mask != NULL && !is_fluid_global(G, mask, i, j)) {
                continue;
            }
            const size_t k = at(G, i, j);
            const double s = cell_max_signal_speed(
                U[0 * G->n + k], U[1 * G->n + k], U[2 * G->n + k], U[3 * G->n + k],
                U[4 * G->n + k], U[5 * G->n + k], U[6 * G->n + k], U[7 * G->n + k], p->gamma);
            m = vmax(m, s);
        }
        row_max[j - G->ng] = m;
    }
    double c_h = 0.0;
    for (int j = 0; j < G->ny; ++j) {
        c_h = vmax(c_h, row_max[j]);
    }
    free(row_max);
    double dt = (c_h <= 0.0) ? HUGE_VAL : p->cfl / (c_h * inv_dx + c_h * inv_dy);
    const double eta_max = max_diffusivity(p);
    if (eta_max > 0.0) {
        const double h = vmin(G->dx, G->dy);
        const double dt_diff = p->cfl * h * h / (2.0 * 2.0 * eta_max);
        dt = vmin(dt, dt_diff);
    }
    *dt_out = dt;
    *ch_out = c_h;
}

int mhdo_cfl(const mhdo_grid* g, const mhdo_params* p, const uint8_t* mask, const double* U,
             double* dt, double* c_h)
{
    geom G;
    if (make_geom(g, &G) != MHDO_OK || p->cfl <= 0.0) {
        return MHDO_EINVAL;
    }
    cfl_dt(&G, p, mask_active(&G, mask) ? mask : NULL, U, dt, c_h);
    return MHDO_OK;
}

/* ---------------------------------------------------------------- spatial operator */

typedef struct {
    double x, y, z;
} vec3;

static vec3 cross3(vec3 a, vec3 b)
{
    vec3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}

static vec3 avg3(double ax, double ay, double az, double bx, double by, double bz)
{
    /* include/mhd/nonideal.hpp:104-107 */
    vec3 r = {0.5 * (ax + bx), 0.5 * (ay + by), 0.5 * (az + bz)};
    return r;
}

/* include/mhd/nonideal.hpp:63-102 */
static vec3 nonideal_e(vec3 J, vec3 B, const mhdo_params* p)
{
    vec3 E = {0.0, 0.0, 0.0};
    if (p->ohmic) {
        E.x += p->eta_ohm * J.x;
        E.y += p->eta_ohm * J.y;
        E.z += p->eta_ohm * J.z;
    }
    if (!(p->hall || p->ambipolar)) {
        return E;
    }
    const double B2 = B.x * B.x + B.y * B.y + B.z * B.z;
    if (B2 < 1.0e-14) {
        return E;
    }
    const vec3 JxB = cross3(J, B);
    if (p->hall) {
        const double invB = 1.0 / sqrt(B2);
        E.x += p->eta_hall * JxB.x * invB;
        E.y += p->eta_hall * JxB.y * invB;
        E.z += p->eta_hall * JxB.z * invB;
    }
    if (p->ambipolar) {
        const vec3 JxBxB = cross3(JxB, B);
        const double invB2 = 1.0 / B2;
        E.x += p->eta_ambipolar * JxBxB.x * invB2;
        E.y += p->eta_ambipolar * JxBxB.y * invB2;
        E.z += p->eta_ambipolar * JxBxB.z * invB2;
    }
    return E;
}

typedef struct {
    double* prim; /* 9 planes, n each: rho, vx, vy, vz, p, bx, by, bz, psi */
    double* J;    /* 3 planes */
    double* fx;   /* 9 planes of ny x (nx + 1) */
    double* fy;   /* 9 planes of (ny + 1) x nx */
} work_t;

void mhdo_nonideal_e(const double* J, const double* B, const mhdo_params* p, double* E)
{
    vec3 j = {J[0], J[1], J[2]}, b = {B[0], B[1], B[2]};
    const vec3 e = nonideal_e(j, b, p);
    E[0] = e.x;
    E[1] = e.y;
    E[2] = e.z;
}

static int work_alloc(const geom* G, work_t* w)
{
    const size_t nfx = (size_t)G->ny * (size_t)(G->nx + 1);
    const size_t nfy = (size_t)(G->ny + 1) * (size_t)G->nx;
    w->prim = (double*)calloc((size_t)NF * G->n, sizeof(double));
    w->J = (double*)calloc(3 * G->n, sizeof(double));
    w->fx = (double*)calloc((size_t)NF * nfx, sizeof(double));
    w->fy = (double*)calloc((size_t)NF * nfy, sizeof(double));
    return (w->prim && w->J && w->fx && w->fy) ? MHDO_OK : MHDO_EINVAL;
}

static void work_free(work_t* w)
{
    free(w->prim);
    free(w->J);
    free(w->fx);
    free(w->fy);
}

static primn load_prim(const geom* G, const double* W, size_t idx, int ydir)
{
    /* include/mhd/kernels/cpu_rows.hpp:40-62 (rotated frame: y-faces swap x and y) */
    primn p;
    p.rho = W[0 * G->n + idx];
    p.vn = W[(ydir ? 2 : 1) * G->n + idx];
    p.vt = W[(ydir ? 1 : 2) * G->n + idx];
    p.vz = W[3 * G->n + idx];
    p.p = W[4 * G->n + idx];
    p.bn = W[(ydir ? 6 : 5) * G->n + idx];
    p.bt = W[(ydir ? 5 : 6) * G->n + idx];
    p.bz = W[7 * G->n + idx];
    p.psi = W[8 * G->n + idx];
    return p;
}

static void store_flux(double* F, size_t plane, size_t k, const fluxn* f, int ydir)
{
    /* include/mhd/kernels/cpu_rows.hpp:64-82 (rotate back to x, y components) */
    F[0 * plane + k] = f->rho;
    F[1 * plane + k] = ydir ? f->mt : f->mn;
    F[2 * plane + k] = ydir ? f->mn : f->mt;
    F[3 * plane + k] = f->mz;
    F[4 * plane + k] = f->e;
    F[5 * plane + k] = ydir ? f->bt : f->bn;
    F[6 * plane + k] = ydir ? f->bn : f->bt;
    F[7 * plane + k] = f->bz;
    F[8 * plane + k] = f->psi;
}

/* include/mhd/rhs.hpp:140-240 (+ fill_primitives :63-70, compute_current nonideal.hpp:30-60,
   add_nonideal_x_row / _y_row rhs.hpp:75-114, assemble_component :116-123). */
static void compute_rhs(const geom* G, const mhdo_params* p, const uint8_t* mask, double c_h,
                        const double* U, double* R, work_t* w)
{
    const double gamma = p->gamma;
    const double inv_gm1 = 1.0 / (gamma - 1.0);
    double* W = w->prim;

    /* Primitives over every cell, ghosts included (cpu_rows.hpp:129-155). */
    #pragma omp parallel for schedule(static)
    for (size_t k = 0; k < G->n; ++k) {
        const double rho = U[0 * G->n + k], mx = U[1 * G->n + k], my = U[2 * G->n + k];
        const double mz = U[3 * G->n + k], e = U[4 * G->n + k];
        const double bx = U[5 * G->n + k], by = U[6 * G->n + k], bz = U[7 * G->n + k];
        const double inv_rho = 1.0 / rho;
        const double ekin = 0.5 * (mx * mx + my * my + mz * mz) * inv_rho;
        const double emag = 0.5 * (bx * bx + by * by + bz * bz);
        W[0 * G->n + k] = rho;
        W[1 * G->n + k] = mx * inv_rho;
        W[2 * G->n + k] = my * inv_rho;
        W[3 * G->n + k] = mz * inv_rho;
        W[4 * G->n + k] = (gamma - 1.0) * (e - ekin - emag);
        W[5 * G->n + k] = bx;
        W[6 * G->n + k] = by;
        W[7 * G->n + k] = bz;
        W[8 * G->n + k] = U[8 * G->n + k];
    }

    const int has_ni = nonideal_any(p);
    if (has_ni) {
        const double inv_2dx = 0.5 / G->dx, inv_2dy = 0.5 / G->dy;
        const int nx = G->nxt;
        const double* bx = W + 5 * G->n;
        const double* by = W + 6 * G->n;
        const double* bz = W + 7 * G->n;
        #pragma omp parallel for schedule(static)
        for (int j = 1; j < G->nyt - 1; ++j) {
            for (int i = 1; i < G->nxt - 1; ++i) {
                const size_t idx = (size_t)j * nx + i;
                const double dbz_dy = (bz[idx + nx] - bz[idx - nx]) * inv_2dy;
                const double dbz_dx = (bz[idx + 1] - bz[idx - 1]) * inv_2dx;
                const double dby_dx = (by[idx + 1] - by[idx - 1]) * inv_2dx;
                const double dbx_dy = (bx[idx + nx] - bx[idx - nx]) * inv_2dy;
                w->J[0 * G->n + idx] = dbz_dy;
                w->J[1 * G->n + idx] = -dbz_dx;
                w->J[2 * G->n + idx] = dby_dx - dbx_dy;
            }
        }
    }

    const size_t pfx = (size_t)G->ny * (size_t)(G->nx + 1);
    const size_t pfy = (size_t)(G->ny + 1) * (size_t)G->nx;
    const double* J = w->J;

    /* x-faces i-1/2 for i = ng .. ng + nx, rows ng .. ng + ny - 1 (cpu_rows.hpp:84-113). */
    #pragma omp parallel for schedule(static)
    for (int jj = 0; jj < G->ny; ++jj) {
        const int j = jj + G->ng;
        for (int k = 0; k <= G->nx; ++k) {
            const int i = G->ng + k;
            const size_t idx = at(G, i, j);
            const primn a = load_prim(G, W, idx - 2, 0), b = load_prim(G, W, idx - 1, 0);
            const primn c = load_prim(G, W, idx, 0), d = load_prim(G, W, idx + 1, 0);
            const fluxn f = muscl_hll_face(p->limiter, &a, &b, &c, &d, gamma, inv_gm1, c_h);
            const size_t fk = (size_t)jj * (size_t)(G->nx + 1) + (size_t)k;
            store_flux(w->fx, pfx, fk, &f, 0);
            if (has_ni) {
                const size_t il = idx - 1, ir = idx;
                const vec3 Jf = avg3(J[il], J[G->n + il], J[2 * G->n + il], J[ir], J[G->n + ir],
                                     J[2 * G->n + ir]);
                const vec3 B = avg3(W[5 * G->n + il], W[6 * G->n + il], W[7 * G->n + il],
                                    W[5 * G->n + ir], W[6 * G->n + ir], W[7 * G->n + ir]);
                const vec3 E = nonideal_e(Jf, B, p);
                w->fx[6 * pfx + fk] += -E.z;
                w->fx[7 * pfx + fk] += E.y;
                w->fx[4 * pfx + fk] += B.y * E.z - B.z * E.y;
            }
        }
    }
    /* y-faces j-1/2 for j = ng .. ng + ny, columns ng .. ng + nx - 1. */
    #pragma omp parallel for schedule(static)
    for (int jj = 0; jj <= G->ny; ++jj) {
        const int j = jj + G->ng;
        for (int k = 0; k < G->nx; ++k) {
            const int i = G->ng + k;
            const size_t idx = at(G, i, j);
            const size_t s = (size_t)G->nxt;
            const primn a = load_prim(G, W, idx - 2 * s, 1), b = load_prim(G, W, idx - s, 1);
            const primn c = load_prim(G, W, idx, 1), d = load_prim(G, W, idx + s, 1);
            const fluxn f = muscl_hll_face(p->limiter, &a, &b, &c, &d, gamma, inv_gm1, c_h);
            const size_t fk = (size_t)jj * (size_t)G->nx + (size_t)k;
            store_flux(w->fy, pfy, fk, &f, 1);
            if (has_ni) {
                const size_t ib = idx - s, it = idx;
                const vec3 Jf = avg3(J[ib], J[G->n + ib], J[2 * G->n + ib], J[it], J[G->n + it],
                                     J[2 * G->n + it]);
                const vec3 B = avg3(W[5 * G->n + ib], W[6 * G->n + ib], W[7 * G->n + ib],
                                    W[5 * G->n + it], W[6 * G->n + it], W[7 * G->n + it]);
                const vec3 E = nonideal_e(Jf, B, p);
                w->fy[5 * pfy + fk] += E.z;
                w->fy[7 * pfy + fk] += -E.x;
                w->fy[4 * pfy + fk] += B.z * E.x - B.x * E.z;
            }
        }
    }

    const double inv_dx = 1.0 / G->dx;
    const double inv_dy = 1.0 / G->dy;
    const double h = vmin(G->dx, G->dy);
    const double psi_damp = (c_h > 0.0 && p->glm_alpha > 0.0) ? (c_h * p->glm_alpha / h) : 0.0;
    #pragma omp parallel for schedule(static)
    for (int jj = 0; jj < G->ny; ++jj) {
        const int j = jj + G->ng;
        for (int k = 0; k < G->nx; ++k) {
            const size_t o = at(G, G->ng + k, j);
            const size_t fx0 = (size_t)jj * (size_t)(G->nx + 1) + (size_t)k;
            const size_t gb = (size_t)jj * (size_t)G->nx + (size_t)k;
            const size_t gt = gb + (size_t)G->nx;
            for (int c = 0; c < NF; ++c) {
                const double* fx = w->fx + (size_t)c * pfx;
                const double* fy = w->fy + (size_t)c * pfy;
                R[(size_t)c * G->n + o] =
                    -(fx[fx0 + 1] - fx[fx0]) * inv_dx - (fy[gt] - fy[gb]) * inv_dy;
            }
            if (psi_damp != 0.0) {
                R[8 * G->n + o] -= psi_damp * U[8 * G->n + o];
            }
            if (mask != NULL && mask[(size_t)jj * (size_t)G->nx + (size_t)k] == 0) {
                for (int c = 0; c < NF; ++c) {
                    R[(size_t)c * G->n + o] = 0.0;
                }
            }
        }
    }
}

int mhdo_rhs(const mhdo_grid* g, const mhdo_params* p, const uint8_t* mask, double c_h,
             const double* U, double* rhs)
{
    geom G;
    work_t w;
    if (make_geom(g, &G) != MHDO_OK) {
        return MHDO_EINVAL;
    }
    if (work_alloc(&G, &w) != MHDO_OK) {
        work_free(&w);
        return MHDO_EINVAL;
    }
    compute_rhs(&G, p, mask_active(&G, mask) ? mask : NULL, c_h, U, rhs, &w);
    work_free(&w);
    return MHDO_OK;
}

/* ---------------------------------------------------------------- time integration */

/* include/mhd/time_integrator.hpp:36-60 with field_xpay / field_ssp_rk2_combine
   (include/mhd/field_ops.hpp:47-63,80-111) over the full array, ghosts included. */
static void ssp_rk2_step(const mhdo_grid* g, const geom* G, const mhdo_params* p, int bc_x,
                         int bc_y, const uint8_t* mask, int walls, double dt, double c_h,
                         double* U, double* Us, double* R, work_t* w)
{
    const size_t tot = (size_t)NF * G->n;
    mhdo_apply_bc(g, bc_x, bc_y, U);
    if (mask != NULL && walls) {
        mhdo_wall_fill(g, mask, p->gamma, U);
    }
    compute_rhs(G, p, mask, c_h, U, R, w);
    #pragma omp parallel for schedule(static)
    for (size_t k = 0; k < tot; ++k) {
        Us[k] = U[k] + dt * R[k];
    }
    mhdo_apply_bc(g, bc_x, bc_y, Us);
    if (mask != NULL && walls) {
        mhdo_wall_fill(g, mask, p->gamma, Us);
    }
    compute_rhs(G, p, mask, c_h, Us, R, w);
    const double half_dt = 0.5 * dt;
    #pragma omp parallel for schedule(static)
    for (size_t k = 0; k < tot; ++k) {
        U[k] = 0.5 * (U[k] + Us[k]) + half_dt * R[k];
    }
}

/* include/mhd/time_integrator.hpp:62-106 */
int mhdo_solve(const mhdo_grid* g, const mhdo_params* p, int bc_x, int bc_y,
               const uint8_t* mask, int reflective_walls, double* U, mhdo_result* out)
{
    geom G;
    if (make_geom(g, &G) != MHDO_OK || p == NULL || U == NULL || out == NULL) {
        return MHDO_EINVAL;
    }
    if ((!p->fixed_steps && p->t_end < 0.0) || p->cfl <= 0.0 || bc_x == MHDO_REFLECTIVE ||
        bc_y == MHDO_REFLECTIVE) {
        return MHDO_EINVAL;
    }
    const uint8_t* active = mask_active(&G, mask) ? mask : NULL;
    const double t_end = p->fixed_steps ? HUGE_VAL : p->t_end;

    const size_t tot = (size_t)NF * G.n;
    double* Us = (double*)calloc(tot, sizeof(double));
    double* R = (double*)calloc(tot, sizeof(double)); /* ghost entries stay 0 */
    work_t w;
    if (Us == NULL || R == NULL || work_alloc(&G, &w) != MHDO_OK) {
        free(Us);
        free(R);
        return MHDO_EINVAL;
    }

    out->t = 0.0;
    out->steps = 0;
    out->c_h = 0.0;
    int rc = MHDO_OK;
    while (out->t < t_end && out->steps < p->max_steps) {
        double dt_cfl, c_h;
        cfl_dt(&G, p, active, U, &dt_cfl, &c_h);
        out->c_h = c_h;
        const double dt = vmin(dt_cfl, t_end - out->t);
        if (!(dt > 0.0)) {
            rc = MHDO_EINVAL; /* ssp_rk2_step requires positive dt (time_integrator.hpp:42-44) */
            break;
        }
        ssp_rk2_step(g, &G, p, bc_x, bc_y, active, reflective_walls, dt, c_h, U, Us, R, &w);
        out->t += dt;
        out->steps += 1;
    }
    if (rc == MHDO_OK && !p->fixed_steps && out->t < t_end && out->steps >= p->max_steps) {
        rc = MHDO_EMAXSTEPS;
    }
    if (rc == MHDO_OK) {
        mhdo_apply_bc(g, bc_x, bc_y, U);
        if (active != NULL && reflective_walls) {
            mhdo_wall_fill(g, active, p->gamma, U);
        }
    }
    work_free(&w);
    free(Us);
    free(R);
    return rc;
}

/* ---------------------------------------------------------------- diagnostics */

int mhdo_diagnostics(const mhdo_grid* g, double gamma, const double* U, mhdo_diag* out)
{
    geom G;
    if (make_geom(g, &G) != MHDO_OK || out == NULL) {
        return MHDO_EINVAL;
    }
    const double cell = G.dx * G.dy;
    const double inv_2dx = 0.5 / G.dx, inv_2dy = 0.5 / G.dy;
    double mass = 0.0, energy = 0.0, dmax = 0.0, d2 = 0.0;
    double rmin = HUGE_VAL, pmin = HUGE_VAL;
    int finite = 1;
    for (int j = G.ng; j < G.ng + G.ny; ++j) {
        for (int i = G.ng; i < G.ng + G.nx; ++i) {
            const size_t k = at(&G, i, j);
            const double rho = U[k], mx = U[G.n + k], my = U[2 * G.n + k], mz = U[3 * G.n + k];
            const double E = U[4 * G.n + k];
            const double bx = U[5 * G.n + k], by = U[6 * G.n + k], bz = U[7 * G.n + k];
            const double e_kin = 0.5 * (mx * mx + my * my + mz * mz) / rho;
            const double e_mag = 0.5 * (bx * bx + by * by + bz * bz);
            const double p = (gamma - 1.0) * (E - e_kin - e_mag);
            rmin = vmin(rmin, rho);
            pmin = vmin(pmin, p);
            /* include/verification/diagnostics.hpp:41-52 */
            mass += rho * cell;
            energy += E * cell;
            if (!isfinite(rho) || !isfinite(p) || !isfinite(E) || !isfinite(bx) ||
                !isfinite(by) || !isfinite(bz)) {
                finite = 0;
            }
            /* include/initial_condition/inititial_condition.hpp:273-287 */
            const double dbx = (U[5 * G.n + at(&G, i + 1, j)] - U[5 * G.n + at(&G, i - 1, j)]) * inv_2dx;
            const double dby = (U[6 * G.n + at(&G, i, j + 1)] - U[6 * G.n + at(&G, i, j - 1)]) * inv_2dy;
            const double dv = dbx + dby;
            dmax = vmax(dmax, fabs(dv));
            d2 += dv * dv;
        }
    }
    out->mass = mass;
    out->energy = energy;
    out->div_b_max = dmax;
    out->div_b_l2 = sqrt(d2 / ((double)G.nx * (double)G.ny));
    out->rho_min = rmin;
    out->p_min = pmin;
    out->finite = finite;
    return MHDO_OK;
}
