/*
 * CPU ORACLE — test infrastructure, not the product.  See lgf_oracle.h.
 *
 * Plain-C restatement of the reference Wilson-flow path.  Every function cites
 * the reference lines it restates.  Wilson loops are written as lattice paths
 * (a sequence of +/- unit steps) rather than as the reference's hand-grouped
 * products; the loop geometry, orientation and weights are the reference's.
 * Built with -ffp-contract=off so no fused multiply-adds change the rounding.
 */
#include "lgf_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double re, im; } cx;
typedef struct { cx m[9]; } su3; /* row-major m[3*r+c] (LGF/Math/SU3_mat.h:15-17) */

static inline cx cx_make(double r, double i) { cx z = {r, i}; return z; }
static inline cx cx_add(cx a, cx b) { return cx_make(a.re + b.re, a.im + b.im); }
static inline cx cx_sub(cx a, cx b) { return cx_make(a.re - b.re, a.im - b.im); }
/* C_double operator* (LGF/Math/C_double.h:46-48) */
static inline cx cx_mul(cx a, cx b) { return cx_make(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static inline cx cx_scale(cx a, double s) { return cx_make(a.re * s, a.im * s); }
static inline cx cx_conj(cx a) { return cx_make(a.re, -a.im); }

static su3 su3_zero(void) { su3 z; memset(&z, 0, sizeof z); return z; }
static su3 su3_mul(const su3* a, const su3* b) { /* SU3_mat.cpp:121-133 */
    su3 o;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            o.m[3 * r + c] = cx_add(cx_add(cx_mul(a->m[3 * r], b->m[c]), cx_mul(a->m[3 * r + 1], b->m[3 + c])),
                                    cx_mul(a->m[3 * r + 2], b->m[6 + c]));
    return o;
}
static su3 su3_adj(const su3* a) {
    su3 o;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) o.m[3 * r + c] = cx_conj(a->m[3 * c + r]);
    return o;
}
static su3 su3_addm(const su3* a, const su3* b) {
    su3 o;
    for (int k = 0; k < 9; ++k) o.m[k] = cx_add(a->m[k], b->m[k]);
    return o;
}
static su3 su3_subm(const su3* a, const su3* b) {
    su3 o;
    for (int k = 0; k < 9; ++k) o.m[k] = cx_sub(a->m[k], b->m[k]);
    return o;
}
static su3 su3_scal(const su3* a, double s) {
    su3 o;
    for (int k = 0; k < 9; ++k) o.m[k] = cx_scale(a->m[k], s);
    return o;
}
static double su3_retr(const su3* a) { return a->m[0].re + a->m[4].re + a->m[8].re; }

static su3 su3_load(const double* p) {
    su3 o;
    for (int k = 0; k < 9; ++k) o.m[k] = cx_make(p[2 * k], p[2 * k + 1]);
    return o;
}
static void su3_store(double* p, const su3* a) {
    for (int k = 0; k < 9; ++k) { p[2 * k] = a->m[k].re; p[2 * k + 1] = a->m[k].im; }
}

/* ---------------------------------------------------------------- lattice */
/* global index, x0 slowest (Lattice.cpp:423-436); periodic torus neighbours
 * (Lattice.cpp:447-459) */
typedef struct { int n[4]; long long stride[4]; long long V; } geom;

static geom geom_make(const int shape[4]) {
    geom g;
    for (int d = 0; d < 4; ++d) g.n[d] = shape[d];
    g.stride[3] = 1;
    g.stride[2] = shape[3];
    g.stride[1] = (long long)shape[3] * shape[2];
    g.stride[0] = (long long)shape[3] * shape[2] * shape[1];
    g.V = g.stride[0] * shape[0];
    return g;
}
static inline long long shift(const geom* g, long long s, int d, int step) {
    long long x = (s / g->stride[d]) % g->n[d];
    long long xn = ((x + step) % g->n[d] + g->n[d]) % g->n[d];
    return s + (xn - x) * g->stride[d];
}
static inline su3 link(const double* U, long long s, int mu) { return su3_load(U + ((s * 4 + mu) * 18)); }

long long lgfo_volume(const int shape[4]) { return (long long)shape[0] * shape[1] * shape[2] * shape[3]; }

/* ------------------------------------------------------------------ staple */
/* A = sum_{nu != mu} [ U_nu(x+mu) (U_nu(x) U_mu(x+nu))^dag + (U_mu(x-nu) U_nu(x-nu+mu))^dag U_nu(x-nu) ]
 * (SU3_field.cpp:519-530) */
static su3 staple(const double* U, const geom* g, long long x, int mu) {
    su3 out = su3_zero();
    long long xpm = shift(g, x, mu, +1);
    for (int nu = 0; nu < 4; ++nu) {
        if (nu == mu) continue;
        long long xpn = shift(g, x, nu, +1), xmn = shift(g, x, nu, -1);
        long long xmnpm = shift(g, xmn, mu, +1);
        su3 a1 = link(U, xpm, nu), a2 = link(U, x, nu), a3 = link(U, xpn, mu);
        su3 t = su3_mul(&a2, &a3);
        su3 td = su3_adj(&t);
        su3 up = su3_mul(&a1, &td);
        su3 b1 = link(U, xmn, mu), b2 = link(U, xmnpm, nu), b3 = link(U, xmn, nu);
        su3 t2 = su3_mul(&b1, &b2);
        su3 t2d = su3_adj(&t2);
        su3 lo = su3_mul(&t2d, &b3);
        out = su3_addm(&out, &up);
        out = su3_addm(&out, &lo);
    }
    return out;
}

void lgfo_staple(const double* U, const int shape[4], long long site, int mu, double out[18]) {
    geom g = geom_make(shape);
    su3 s = staple(U, &g, site, mu);
    su3_store(out, &s);
}

/* Z = -1/2 [ (W - W^dag) - 1/3 Tr(W - W^dag) ],  W = U_mu(x) A  (Wilson.cpp:55-71) */
static su3 flow_gradient(const double* U, const geom* g, long long x, int mu) {
    su3 u = link(U, x, mu);
    su3 a = staple(U, g, x, mu);
    su3 w = su3_mul(&u, &a);
    su3 wd = su3_adj(&w);
    su3 t = su3_subm(&w, &wd);
    cx tr = cx_add(cx_add(t.m[0], t.m[4]), t.m[8]);
    tr = cx_scale(tr, 1.0 / 3.0);
    t.m[0] = cx_sub(t.m[0], tr);
    t.m[4] = cx_sub(t.m[4], tr);
    t.m[8] = cx_sub(t.m[8], tr);
    return su3_scal(&t, -0.5);
}

void lgfo_flow_gradient(const double* U, const int shape[4], long long site, int mu, double out[18]) {
    geom g = geom_make(shape);
    su3 z = flow_gradient(U, &g, site, mu);
    su3_store(out, &z);
}

/* --------------------------------------------------------- exponential */
/* exp(iP) for anti-Hermitian traceless iP by the Cayley-Hamilton method of
 * Morningstar & Peardon (hep-lat/0311018), with the reference's branch
 * structure and thresholds (SU3_mat.cpp:216-289): Q = -i iP, c0 = ReTr(Q^3)/3,
 * c1 = ReTr(Q^2)/2, analytic f_j when c1 > 1e-4 (eqs. 23-34, conjugation rule
 * for c0 < 0), series f_j otherwise; xi0 by series when |w| <= 0.05.
 * Release-build semantics: no clamp on the acos argument. */
static su3 exp_iP(const su3* iP) {
    su3 Q;
    for (int k = 0; k < 9; ++k) Q.m[k] = cx_make(iP->m[k].im, -iP->m[k].re); /* timesMinusI */
    su3 Q2 = su3_mul(&Q, &Q);
    su3 Q3 = su3_mul(&Q, &Q2);
    double c0 = su3_retr(&Q3) / 3.0;
    double c1 = su3_retr(&Q2) / 2.0;
    cx f0, f1, f2;
    if (c1 > 0.0001) {
        double c1s = sqrt(c1);
        double r = fabs(c0) / (2.0 * pow(c1 / 3.0, 1.5));
        double th3 = acos(r) / 3.0;
        double u = sqrt(1.0 / 3.0) * c1s * cos(th3);
        double w = c1s * sin(th3);
        double u2 = u * u, w2 = w * w;
        double uc = cos(u), us = sin(u), wc = cos(w);
        double xi0 = fabs(w) > 0.05 ? sin(w) / w : 1.0 - w2 * (1.0 - w2 * (1 - w2 / 42.0) / 20.0) / 6.0;
        double div = 1.0 / (9.0 * u2 - w2);
        cx e2iu = cx_make(2.0 * uc * uc - 1.0, 2.0 * uc * us);
        cx emiu = cx_make(uc, -us);
        cx h0 = cx_add(cx_scale(e2iu, u2 - w2), cx_mul(emiu, cx_make(8.0 * u2 * wc, 2.0 * u * (3.0 * u2 + w2) * xi0)));
        cx h1 = cx_sub(cx_scale(e2iu, 2.0 * u), cx_mul(emiu, cx_make(2.0 * u * wc, (w2 - 3.0 * u2) * xi0)));
        cx h2 = cx_sub(e2iu, cx_mul(emiu, cx_make(wc, 3.0 * u * xi0)));
        f0 = cx_scale(h0, div);
        f1 = cx_scale(h1, div);
        f2 = cx_scale(h2, div);
        if (c0 < 0.0) {
            f0 = cx_conj(f0);
            f1 = cx_scale(cx_conj(f1), -1.0);
            f2 = cx_conj(f2);
        }
    } else {
        double c02 = c0 * c0;
        f0 = cx_make(1.0 - c02 / 720.0, -c0 * (1.0 - c1 * (1 - c1 / 42.0) / 20.0) / 6.0);
        f1 = cx_make(c0 * (1.0 - c1 * (1.0 - 3.0 * c1 / 112.0) / 15.0) / 24.0,
                     1.0 - c1 * (1.0 - c1 * (1 - c1 / 42.0) / 20.0) / 6.0 - c02 / 5040.0);
        f2 = cx_make((-1.0 + c1 * (1.0 - c1 * (1.0 - c1 / 56.0) / 30.0) / 12.0 + c02 / 20160.0) / 2.0,
                     (c0 * (1.0 - c1 * (1.0 - c1 / 48.0) / 21.0) / 60.0) / 2.0);
    }
    su3 out;
    for (int k = 0; k < 9; ++k) out.m[k] = cx_add(cx_mul(Q.m[k], f1), cx_mul(Q2.m[k], f2));
    out.m[0] = cx_add(out.m[0], f0);
    out.m[4] = cx_add(out.m[4], f0);
    out.m[8] = cx_add(out.m[8], f0);
    return out;
}

void lgfo_exp_iP(const double iP[18], double out[18]) {
    su3 a = su3_load(iP);
    su3 e = exp_iP(&a);
    su3_store(out, &e);
}

void lgfo_exp_iP_many(const double* iP, double* out, long long n) {
    for (long long i = 0; i < n; ++i) lgfo_exp_iP(iP + 18 * i, out + 18 * i);
}

/* ------------------------------------------------------------- RK3 step */
static void gradient_field(const double* U, const geom* g, double* Z) {
    for (long long x = 0; x < g->V; ++x)
        for (int mu = 0; mu < 4; ++mu) {
            su3 z = flow_gradient(U, g, x, mu);
            su3_store(Z + (x * 4 + mu) * 18, &z);
        }
}

/* Luscher RK3 (GradientFlow.cpp:22-54):
 *   W1 = exp(eps/4 Z0) W0
 *   W2 = exp(eps (8/9 Z1 - 17/36 Z0)) W1
 *   W3 = exp(eps (3/4 Z2 - 8/9 Z1 + 17/36 Z0)) W2 */
void lgfo_rk3_step(double* U, const int shape[4], double eps, double* scratch) {
    geom g = geom_make(shape);
    const long long nl = g.V * 4;
    double* Z0 = scratch;
    double* Z1 = scratch + nl * 18;
    double* Z2 = scratch + 2 * nl * 18;
    for (int stage = 0; stage < 3; ++stage) {
        double* Zs = stage == 0 ? Z0 : (stage == 1 ? Z1 : Z2);
        gradient_field(U, &g, Zs);
        for (long long l = 0; l < nl; ++l) {
            su3 z0 = su3_load(Z0 + l * 18), X;
            if (stage == 0) {
                X = su3_scal(&z0, 0.25 * eps);
            } else if (stage == 1) {
                su3 z1 = su3_load(Z1 + l * 18);
                su3 a = su3_scal(&z1, 8.0 / 9.0), b = su3_scal(&z0, 17.0 / 36.0);
                su3 c = su3_subm(&a, &b);
                X = su3_scal(&c, eps);
            } else {
                su3 z1 = su3_load(Z1 + l * 18), z2 = su3_load(Z2 + l * 18);
                su3 a = su3_scal(&z2, 3.0 / 4.0), b = su3_scal(&z1, 8.0 / 9.0), c = su3_scal(&z0, 17.0 / 36.0);
                su3 d = su3_subm(&a, &b);
                su3 e = su3_addm(&d, &c);
                X = su3_scal(&e, eps);
            }
            su3 ex = exp_iP(&X);
            su3 u = su3_load(U + l * 18);
            su3 un = su3_mul(&ex, &u);
            su3_store(U + l * 18, &un);
        }
    }
}

/* ------------------------------------------------------- Wilson loops */
/* Product of links along a path from x: a step +d multiplies U_d(y) and moves
 * y -> y+d; a step -d moves y -> y-d and multiplies U_d(y)^dag. */
static su3 path_product(const double* U, const geom* g, long long x, const int* steps, int n) {
    long long y = x;
    su3 acc;
    for (int i = 0; i < n; ++i) {
        int d = abs(steps[i]) - 1;
        su3 l;
        if (steps[i] > 0) {
            l = link(U, y, d);
            y = shift(g, y, d, +1);
        } else {
            y = shift(g, y, d, -1);
            su3 t = link(U, y, d);
            l = su3_adj(&t);
        }
        if (i == 0) acc = l;
        else acc = su3_mul(&acc, &l);
    }
    return acc;
}

/* Sum of the four a x b rectangular loops (a links along mu, b along nu) that
 * start and end at x, one per quadrant, in the orientation the reference uses
 * for every clover-type average (SU3_field.cpp:550-560, 606-631, 654-694,
 * 723-775):  (+nu^b +mu^a -nu^b -mu^a), (+mu^a -nu^b -mu^a +nu^b),
 *            (-mu^a +nu^b +mu^a -nu^b), (-nu^b -mu^a +nu^b +mu^a). */
static su3 four_leaves(const double* U, const geom* g, long long x, int mu, int nu, int a, int b) {
    const int M = mu + 1, N = nu + 1;
    int st[16];
    su3 sum = su3_zero();
    const int seg[4][4][2] = {{{+N, b}, {+M, a}, {-N, b}, {-M, a}},
                              {{+M, a}, {-N, b}, {-M, a}, {+N, b}},
                              {{-M, a}, {+N, b}, {+M, a}, {-N, b}},
                              {{-N, b}, {-M, a}, {+N, b}, {+M, a}}};
    for (int leaf = 0; leaf < 4; ++leaf) {
        int n = 0;
        for (int s = 0; s < 4; ++s)
            for (int r = 0; r < seg[leaf][s][1]; ++r) st[n++] = seg[leaf][s][0];
        su3 w = path_product(U, g, x, st, n);
        sum = su3_addm(&sum, &w);
    }
    return sum;
}

/* F = -i/2 [ (C - C^dag) - 1/3 Tr(C - C^dag) ]  (SU3_field.cpp:575-579) */
static su3 project_F(const su3* C) {
    su3 cd = su3_adj(C);
    su3 t = su3_subm(C, &cd);
    cx tr = cx_scale(cx_add(cx_add(t.m[0], t.m[4]), t.m[8]), 1.0 / 3.0);
    t.m[0] = cx_sub(t.m[0], tr);
    t.m[4] = cx_sub(t.m[4], tr);
    t.m[8] = cx_sub(t.m[8], tr);
    su3 o;
    for (int k = 0; k < 9; ++k) o.m[k] = cx_make(0.5 * t.m[k].im, -0.5 * t.m[k].re);
    return o;
}

static su3 clover_F(const double* U, const geom* g, long long x, int mu, int nu) {
    su3 w = four_leaves(U, g, x, mu, nu, 1, 1);
    su3 c = su3_scal(&w, 0.25);
    return project_F(&c);
}

/* F^ = 19/9 F[C11] + 1/36 F[C22] - 32/45 F[C12] + 1/15 F[C13]  (SU3_field.cpp:588-597);
 * C22 = 1/4 (2x2 leaves), C12 = 1/8 (1x2 + 2x1 leaves), C13 = 1/8 (1x3 + 3x1 leaves) */
static su3 improved_F(const double* U, const geom* g, long long x, int mu, int nu) {
    su3 c11 = four_leaves(U, g, x, mu, nu, 1, 1);
    su3 c22 = four_leaves(U, g, x, mu, nu, 2, 2);
    su3 t12 = four_leaves(U, g, x, mu, nu, 1, 2), w12 = four_leaves(U, g, x, mu, nu, 2, 1);
    su3 t13 = four_leaves(U, g, x, mu, nu, 1, 3), w13 = four_leaves(U, g, x, mu, nu, 3, 1);
    c11 = su3_scal(&c11, 0.25);
    c22 = su3_scal(&c22, 0.25);
    t12 = su3_scal(&t12, 1.0 / 8.0);
    w12 = su3_scal(&w12, 1.0 / 8.0);
    t13 = su3_scal(&t13, 1.0 / 8.0);
    w13 = su3_scal(&w13, 1.0 / 8.0);
    su3 c12 = su3_addm(&t12, &w12), c13 = su3_addm(&t13, &w13);
    su3 f11 = project_F(&c11), f22 = project_F(&c22), f12 = project_F(&c12), f13 = project_F(&c13);
    su3 o;
    for (int k = 0; k < 9; ++k) {
        cx v = cx_scale(f11.m[k], 19.0 / 9.0);
        v = cx_add(v, cx_scale(f22.m[k], 1.0 / 36.0));
        v = cx_add(v, cx_scale(f12.m[k], -32.0 / 45.0));
        v = cx_add(v, cx_scale(f13.m[k], 1.0 / 15.0));
        o.m[k] = v;
    }
    return o;
}

void lgfo_clover_F(const double* U, const int shape[4], long long site, int mu, int nu, double out[18]) {
    geom g = geom_make(shape);
    su3 f = clover_F(U, &g, site, mu, nu);
    su3_store(out, &f);
}

void lgfo_improved_F(const double* U, const int shape[4], long long site, int mu, int nu, double out[18]) {
    geom g = geom_make(shape);
    su3 f = improved_F(U, &g, site, mu, nu);
    su3_store(out, &f);
}

static double retr_prod(const su3* a, const su3* b) {
    su3 p = su3_mul(a, b);
    return su3_retr(&p);
}

/* e(x) = sum_{mu<nu} ReTr(F F) with the clover F (EnergyDensity.cpp:13-20);
 * q(x) = ReTr(F^32 F^01) + ReTr(F^31 F^20) + ReTr(F^30 F^12) with the improved F
 * (TopologicalCharge.cpp:11-16). */
static void site_densities(const double* U, const geom* g, long long x, double* e, double* q) {
    double es = 0.0;
    for (int mu = 0; mu < 4; ++mu)
        for (int nu = mu + 1; nu < 4; ++nu) {
            su3 f = clover_F(U, g, x, mu, nu);
            es += retr_prod(&f, &f);
        }
    su3 f32 = improved_F(U, g, x, 3, 2), f01 = improved_F(U, g, x, 0, 1);
    su3 f31 = improved_F(U, g, x, 3, 1), f20 = improved_F(U, g, x, 2, 0);
    su3 f30 = improved_F(U, g, x, 3, 0), f12 = improved_F(U, g, x, 1, 2);
    double qs = 0.0;
    qs += retr_prod(&f32, &f01);
    qs += retr_prod(&f31, &f20);
    qs += retr_prod(&f30, &f12);
    *e = es;
    *q = qs;
}

void lgfo_site_densities(const double* U, const int shape[4], double* e_site, double* q_site) {
    geom g = geom_make(shape);
    for (long long x = 0; x < g.V; ++x) site_densities(U, &g, x, &e_site[x], &q_site[x]);
}

static void measure(const double* U, const geom* g, double* E, double* Q, double* E_slice, double* Q_slice) {
    static const double PI = 3.14159265358979323846;
    const long long vs = g->V / g->n[0];
    double Es = 0.0, Qs = 0.0;
    for (int t = 0; t < g->n[0]; ++t) {
        double et = 0.0, qt = 0.0;
        for (long long i = 0; i < vs; ++i) {
            double e, q;
            site_densities(U, g, t * vs + i, &e, &q);
            et += e;
            qt += q;
        }
        if (E_slice) E_slice[t] = et / (double)vs;
        if (Q_slice) Q_slice[t] = qt * (1.0 / (4.0 * PI * PI));
        Es += et;
        Qs += qt;
    }
    if (E) *E = Es * (1.0 / (double)g->V);      /* EnergyDensity.cpp:26 */
    if (Q) *Q = Qs * (1.0 / (4.0 * PI * PI));  /* TopologicalCharge.cpp:21 */
}

double lgfo_energy_density(const double* U, const int shape[4], double* per_slice) {
    geom g = geom_make(shape);
    double E;
    measure(U, &g, &E, NULL, per_slice, NULL);
    return E;
}

double lgfo_topological_charge(const double* U, const int shape[4], double* per_slice) {
    geom g = geom_make(shape);
    double Q;
    measure(U, &g, NULL, &Q, NULL, per_slice);
    return Q;
}

int lgfo_flow(double* U, const int shape[4], double eps, int nsteps, int meas_every, double t0,
              double* t_out, double* E_out, double* Q_out) {
    geom g = geom_make(shape);
    double* scratch = (double*)malloc(sizeof(double) * 3 * 18 * 4 * (size_t)g.V);
    if (!scratch) return -1;
    int m = 0;
    double t = t0;
    measure(U, &g, &E_out[m], &Q_out[m], NULL, NULL);
    t_out[m++] = t;
    for (int s = 1; s <= nsteps; ++s) {
        lgfo_rk3_step(U, shape, eps, scratch);
        t += eps;
        if (meas_every > 0 && s % meas_every == 0) {
            measure(U, &g, &E_out[m], &Q_out[m], NULL, NULL);
            t_out[m++] = t;
        }
    }
    free(scratch);
    return m;
}

/* ---------------------------------------------------------- generator G */
/* splitmix64 finaliser (Steele, Lea & Flood, OOPSLA 2014) as a counter hash */
static inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
static inline double unit_open(uint64_t seed, uint64_t ctr) {
    uint64_t r = mix64(seed ^ mix64(ctr));
    return ((double)(r >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

void lgfo_generate_G(const int shape[4], unsigned long long seed, double scale, double* U) {
    static const double TWO_PI = 6.28318530717958647692;
    const double inv_sqrt3 = 1.0 / sqrt(3.0);
    long long nl = lgfo_volume(shape) * 4;
    for (long long l = 0; l < nl; ++l) {
        double h[8];
        for (int a = 0; a < 8; ++a) {
            uint64_t c = (uint64_t)l * 8u + (uint64_t)a;
            double u1 = unit_open(seed, 2 * c), u2 = unit_open(seed, 2 * c + 1);
            h[a] = sqrt(-2.0 * log(u1)) * cos(TWO_PI * u2);
        }
        /* H = sum_a h_a lambda_a / 2 */
        su3 H = su3_zero();
        H.m[1] = cx_make(0.5 * h[0], -0.5 * h[1]);
        H.m[3] = cx_make(0.5 * h[0], 0.5 * h[1]);
        H.m[2] = cx_make(0.5 * h[3], -0.5 * h[4]);
        H.m[6] = cx_make(0.5 * h[3], 0.5 * h[4]);
        H.m[5] = cx_make(0.5 * h[5], -0.5 * h[6]);
        H.m[7] = cx_make(0.5 * h[5], 0.5 * h[6]);
        H.m[0] = cx_make(0.5 * h[2] + 0.5 * inv_sqrt3 * h[7], 0.0);
        H.m[4] = cx_make(-0.5 * h[2] + 0.5 * inv_sqrt3 * h[7], 0.0);
        H.m[8] = cx_make(-inv_sqrt3 * h[7], 0.0);
        su3 X; /* X = i * scale * H */
        for (int k = 0; k < 9; ++k) X.m[k] = cx_make(-scale * H.m[k].im, scale * H.m[k].re);
        su3 e = exp_iP(&X);
        su3_store(U + l * 18, &e);
    }
}

void lgfo_unitarity(const double* U, long long nlinks, double* max_unit_err, double* max_det_err) {
    double mu = 0.0, md = 0.0;
    for (long long l = 0; l < nlinks; ++l) {
        su3 u = su3_load(U + 18 * l);
        su3 ud = su3_adj(&u);
        su3 p = su3_mul(&ud, &u);
        double s = 0.0;
        for (int k = 0; k < 9; ++k) {
            double re = p.m[k].re - ((k % 4) == 0 ? 1.0 : 0.0);
            s += re * re + p.m[k].im * p.m[k].im;
        }
        s = sqrt(s);
        cx d = cx_sub(cx_mul(u.m[0], cx_sub(cx_mul(u.m[4], u.m[8]), cx_mul(u.m[5], u.m[7]))),
                      cx_mul(u.m[1], cx_sub(cx_mul(u.m[3], u.m[8]), cx_mul(u.m[5], u.m[6]))));
        d = cx_add(d, cx_mul(u.m[2], cx_sub(cx_mul(u.m[3], u.m[7]), cx_mul(u.m[4], u.m[6]))));
        double de = hypot(d.re - 1.0, d.im);
        if (s > mu) mu = s;
        if (de > md) md = de;
    }
    *max_unit_err = mu;
    *max_det_err = md;
}
